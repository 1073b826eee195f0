// Kernel (c), two-stage form: reduction of the Hermitian BSE matrix to real symmetric
// tridiagonal form in two steps, dense -> band (bandwidth b = 32) -> tridiagonal.
//
// Reference: the dense ZHEEV('V','U') of bsesolver (subprograms/bse_solver-tool-diel.f90:
// 485-492) and ZHEEV('N','U') of bsebnds (bse_kpath-tool.f90:384-387).  The one-stage
// reduction (tridiag.cu) streams the whole trailing matrix once per column in a Hermitian
// matrix-vector product, so half of its flops run at HBM speed.  Here:
//
// Stage 1 (dense -> band), per panel of b columns j0..j0+b-1 with k0 = j0 + b:
//   (1) k_panel_qr: Householder QR of the panel A[k0:N, j0:j0+b] (ZLARFG reflectors, one
//       cooperative launch whose CTAs keep their row slices in shared memory, two bounded grid
//       barriers per column); the T factor of the block reflector Q = I - V T V^H; the velocity
//       vectors g <- Q^T g = g - conj(V) T^T (V^T g).
//   (2) k_hemm2: X = A22 V on the FP64 tensor cores (mma.sync m16n8k16), A22 = A[k0:N, k0:N]
//       read once from its stored lower triangle (tiles above the diagonal are read transposed
//       and conjugated, the diagonal tiles from a symmetrised copy), split over K into
//       deterministic partial sums.
//   (3) k_xreduce / k_mform / k_wform: X <- X T, M = T^H V^H X, W = X - 1/2 V M.
//   (4) k_her2k (tridiag.cu): A22 -= V W^H + W V^H, so that A22 <- Q^H A22 Q.
//   Both large products are GEMM-shaped, so the stage runs at tensor-core speed where the
//   one-stage mat-vec runs at HBM speed.
// Stage 2 (band -> tridiagonal, bulge chasing) is in the second half of this file.
// The oscillator strengths need only A^T h = Z^T (Q^T h), so no O(N^3) back-transform is formed.
#include <cfloat>

#include "common.cuh"

#include <algorithm>
#include <string>

// implemented in tridiag.cu
int launch_her2k_v(wtbg_ctx* ctx, double2* A, long long N, const double2* Wp, const double2* V, long long vld, int vc0,
                   int jb, long long k0);

namespace {

constexpr int BW = 32;            // band width b of the two-stage reduction (= WTBG_PANEL)
constexpr int PQ_THREADS = 256;   // threads of the panel QR kernel
constexpr int PQ_MAXG = 160;      // largest panel-QR grid (one CTA per SM; the host checks)
constexpr int NGMAX = 10;         // velocity vectors carried through (x, y, z, sp, sm [, times f])

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

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned int* p, unsigned int v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
constexpr unsigned long long kWaitNs = 2000000000ull;   // 2 s bound on every spin wait

// Bounded acquire-wait until *p >= need.  The error flag and the clock are read every 64 polls,
// so that a detection costs one L2 round trip; after 2 s, or when another CTA or warp has
// failed, the flag is set and the wait reports failure.
__device__ __forceinline__ bool wait_at_least(const unsigned int* p, unsigned int need, int* err) {
  unsigned int spins = 0;
  unsigned long long t0 = 0;
  while (ld_acquire(p) < need) {
    if ((++spins & 63u) == 0u) {
      if (t0 == 0) t0 = globaltimer();
      if (ld_acquire(reinterpret_cast<unsigned int*>(err)) != 0u || globaltimer() - t0 > kWaitNs) {
        atomicExch(err, 1);
        return false;
      }
    }
  }
  return true;
}

// Grid barrier among the co-resident CTAs of a cooperative launch.  Each launch has its own
// arrival counter, zeroed before the launch; barrier k of the launch is passed when the counter
// reaches k * gridDim.x.  Thread 0 arrives with a release reduction (no returned value, no reset
// step) and polls with acquire loads; the CTA barrier around it orders the other threads' memory
// operations (as in a cooperative-groups grid sync).  The wait is bounded (2 s of %globaltimer);
// on time-out (or when another CTA has already failed) the CTA sets *err and the barrier reports
// failure, after which every CTA leaves the kernel.
__device__ bool grid_sync(unsigned int* cnt, unsigned int target, int* err) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(cnt) : "memory");
    s_ok = wait_at_least(cnt, target, err) ? 1 : 0;
  }
  __syncthreads();
  return s_ok != 0;
}

// ----------------------------------------------------------------------------- stage 1
// Panel QR.  CTA c owns rows [k0 + c*R, k0 + min((c+1)*R, m)) of the panel, kept in shared
// memory as P[col][row] (row fastest).  Per column p: ZLARFG from the grid-reduced norm (every
// CTA sums the same partials in the same order, so all hold identical scalars), then the
// reflector is applied to the panel's remaining columns with grid-reduced dot products.
// The column step is one latency chain (grid barrier, reduction of the CTAs' partials, scalars,
// update, next partials), so every part of it uses all threads: 8 threads per column reduce the
// partials and form the next ones (fixed order, width-8 shuffle tree), every thread evaluates
// the reflector scalars itself, and the update runs over (row, 8-column chunk) items.
struct PanelArgs {
  double2* A;
  long long N;
  int j0, k0, jb;      // panel columns j0 .. j0+jb-1, first panel row k0
  int nref;            // reflectors: min(jb, N - k0)
  int R;               // rows per CTA
  int RS;              // column stride of the panel slice in shared memory (R rounded up to odd)
  double2* Vp;         // [32][N] dense V (rows k0.. written, explicit unit and zeros)
  double2* Tout;       // [32][32] column-major T factor
  double2* g;          // [ng][N]
  int ng;
  double* partN;       // [grid]
  double2* partW;      // [2][grid][32] partial norms (column p) and unscaled dots, by parity of p
  double2* partG;      // [grid][32*32]
  double2* partVg;     // [grid][32*NGMAX]
  double2* alpha;      // [2][32] posted row k0 + p (alpha = its column-p entry), by parity of p
  unsigned int* cnt;   // this launch's grid-barrier arrival counter (zero at launch)
  int* err;
};

__device__ __forceinline__ double2 ldcg2(const double2* p) { return __ldcg(p); }

__global__ void __launch_bounds__(PQ_THREADS, 1) k_panel_qr(PanelArgs a) {
  extern __shared__ __align__(16) double2 P[];   // [jb][R]
  __shared__ double2 s_tau[BW];
  __shared__ double2 s_w[BW];
  __shared__ double2 s_S[BW];    // grid-reduced S_q of the current column (q >= p)
  __shared__ double2 s_al[BW];   // posted row k0 + p
  __shared__ double2 s_T[BW * BW];
  __shared__ double2 s_y[BW * NGMAX];
  const int tid = threadIdx.x;
  const int R = a.R, RS = a.RS, jb = a.jb;   // rows per CTA; shared-memory column stride (odd)
  const long long N = a.N;
  const int G = (int)gridDim.x;
  const long long rbeg = (long long)a.k0 + (long long)blockIdx.x * R;
  const long long rend = min((long long)a.k0 + (long long)(blockIdx.x + 1) * R, N);
  const int nr = (int)max(0LL, rend - rbeg);
  unsigned int nbar = 0;
  auto sync_grid = [&]() -> bool {
    ++nbar;
    return grid_sync(a.cnt, nbar * (unsigned int)G, a.err);
  };
  for (int q = 0; q < jb; ++q)
    for (int i = tid; i < R; i += PQ_THREADS)
      P[(size_t)q * RS + i] = (i < nr) ? a.A[(rbeg + i) + (long long)(a.j0 + q) * N] : make_double2(0, 0);
  __syncthreads();

  // width-8 sum over the aligned lane groups of 8 (every lane of a group ends with the same sum)
  auto sum8 = [](double2 v) {
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
      v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
      v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
  };
  const int qq = tid >> 3, sl = tid & 7;   // column offset and slice of the 8-thread groups

  // Partials of column p over the own rows below row k0 + p, one reduction for both the norm
  // and the unscaled dot products: S_q = sum_{r > k0+p} conj(P[r,p]) P[r,q] for q = p .. jb-1
  // (S_p = |x|^2); thread slice sl takes the rows i = sl (mod 8).  The owner of row k0 + p
  // posts that row (alpha = P[k0+p, p] and P[k0+p, q]).  Buffers alternate with the parity of
  // p: a CTA writes the partials of column p+1 while others may still read those of p, but
  // never those of p+2 before everyone passed the barrier of p+1.
  auto partials = [&](int p) {
    const long long rp = (long long)a.k0 + p;
    const int buf = p & 1;
    double2 sacc = make_double2(0, 0);
    if (qq < jb - p) {
      const double2* Pp = P + (size_t)p * RS;
      const double2* Pq = P + (size_t)(p + qq) * RS;
      const int i0 = (int)max(0LL, rp + 1 - rbeg);
      for (int i = i0 + ((sl - i0) & 7); i < nr; i += 8) sacc = cadd(sacc, cmulc(Pp[i], Pq[i]));
    }
    sacc = sum8(sacc);
    if (qq < jb - p && sl == 0) a.partW[((size_t)buf * G + blockIdx.x) * BW + p + qq] = sacc;
    if (rp >= rbeg && rp < rend)
      for (int q = p + tid; q < jb; q += PQ_THREADS) a.alpha[buf * BW + q] = P[(size_t)q * RS + (rp - rbeg)];
  };

  partials(0);
  for (int p = 0; p < a.nref; ++p) {
    if (!sync_grid()) return;
    const long long rp = (long long)a.k0 + p;
    const int buf = p & 1;
    // grid reduction of S_q (q = p + qq): slice sl sums the CTAs c = sl (mod 8) in order, its
    // (at most PQ_MAXG / 8) loads issued together
    {
      double2 sacc = make_double2(0, 0);
      if (qq < jb - p) {
        double2 pv[PQ_MAXG / 8];
#pragma unroll
        for (int u = 0; u < PQ_MAXG / 8; ++u) {
          const int c = sl + 8 * u;
          pv[u] = (c < G) ? ldcg2(a.partW + ((size_t)buf * G + c) * BW + p + qq) : make_double2(0, 0);
        }
#pragma unroll
        for (int u = 0; u < PQ_MAXG / 8; ++u)
          if (sl + 8 * u < G) sacc = cadd(sacc, pv[u]);
      }
      sacc = sum8(sacc);
      if (qq < jb - p) {
        if (sl == 0) s_S[p + qq] = sacc;
        else if (sl == 1) s_al[p + qq] = ldcg2(a.alpha + buf * BW + p + qq);
      }
    }
    __syncthreads();
    // ZLARFG scalars, evaluated by every thread from the same shared values
    double2 tau, scal;
    double beta;
    {
      const double xn2 = s_S[p].x;
      const double2 al = s_al[p];
      if (xn2 == 0.0 && al.y == 0.0) {
        tau = make_double2(0, 0);
        scal = make_double2(0, 0);
        beta = al.x;
      } else {
        beta = -copysign(sqrt(al.x * al.x + al.y * al.y + xn2), al.x);
        tau = make_double2((beta - al.x) / beta, -al.y / beta);
        const double2 den = make_double2(al.x - beta, al.y);
        const double dd = den.x * den.x + den.y * den.y;
        scal = make_double2(den.x / dd, -den.y / dd);
      }
    }
    if (tid == 0) s_tau[p] = tau;
    // P[r,q] -= conj(tau) v_r w_q (r >= k0+p, q > p), with v_r = P[r,p] scal (v = 1 at row
    // k0+p) and w_q = sum_{r >= k0+p} conj(v_r) P[r,q] = P[k0+p, q] + conj(scal) S_q
    {
      const double2 ct = cconj(tau);
      const int nch = (jb - p - 1 + 7) >> 3;
      for (int it = tid; it < nr * nch; it += PQ_THREADS) {
        const int i = it % nr, ch = it / nr;
        const long long r = rbeg + i;
        if (r < rp) continue;
        const double2 v = (r == rp) ? make_double2(1.0, 0.0) : cmul(P[(size_t)p * RS + i], scal);
        const double2 cv = cmul(ct, v);
        const int q0 = p + 1 + ch * 8, q1 = min(q0 + 8, jb);
        for (int q = q0; q < q1; ++q) {
          const double2 wq = cadd(s_al[q], cmul(cconj(scal), s_S[q]));
          P[(size_t)q * RS + i] = csub(P[(size_t)q * RS + i], cmul(cv, wq));
        }
      }
    }
    __syncthreads();
    // column p becomes v (beta on row k0+p), then the partials of column p+1
    for (int i = tid; i < nr; i += PQ_THREADS) {
      const long long r = rbeg + i;
      if (r == rp) P[(size_t)p * RS + i] = make_double2(beta, 0.0);
      else if (r > rp) P[(size_t)p * RS + i] = cmul(P[(size_t)p * RS + i], scal);
    }
    if (p + 1 < a.nref) partials(p + 1);
  }
  __syncthreads();
  // write back: A keeps R (rows <= k0+q) and v below; Vp gets V with its unit and zeros
  auto vval = [&](int q, int i) -> double2 {
    const long long r = rbeg + i, rq = (long long)a.k0 + q;
    if (q >= a.nref || r < rq) return make_double2(0, 0);
    if (r == rq) return make_double2(1.0, 0.0);
    return P[(size_t)q * RS + i];
  };
  for (int q = 0; q < jb; ++q)
    for (int i = tid; i < nr; i += PQ_THREADS) {
      a.A[(rbeg + i) + (long long)(a.j0 + q) * N] = P[(size_t)q * RS + i];
      a.Vp[(rbeg + i) + (long long)q * N] = vval(q, i);
    }
  // P becomes the explicit V (unit on row k0+q, zeros above it and in columns >= nref), so that
  // the Gram and velocity sums below run without branches
  __syncthreads();
  const int nref = a.nref;
  for (int q = 0; q < jb; ++q)
    for (int i = tid; i < nr; i += PQ_THREADS) {
      const long long r = rbeg + i, rq = (long long)a.k0 + q;
      if (q >= nref || r < rq) P[(size_t)q * RS + i] = make_double2(0, 0);
      else if (r == rq) P[(size_t)q * RS + i] = make_double2(1.0, 0.0);
    }
  __syncthreads();
  // Gram partial V^H V over the own rows: thread t sums the four entries (t mod 32, t/32 + 8k) in
  // one pass (one column per lane, the odd stride keeps the 32 lanes on distinct banks; the
  // other column is a broadcast), rows in order
  {
    const int qi = tid & (BW - 1), qj0 = tid >> 5;
    double2 s4[4] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    const double2* Pi = P + (size_t)qi * RS;
    for (int i = 0; i < nr; ++i) {
      const double2 vi = Pi[i];
#pragma unroll
      for (int k = 0; k < 4; ++k) s4[k] = cadd(s4[k], cmulc(vi, P[(size_t)(qj0 + 8 * k) * RS + i]));
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) a.partG[(size_t)blockIdx.x * BW * BW + tid + PQ_THREADS * k] = s4[k];
  }
  // V^T g over the own rows, rows in order; the loads of 16 rows are issued together
  for (int e = tid; e < BW * a.ng; e += PQ_THREADS) {
    const int q = e % BW, al = e / BW;
    const double2* gp = a.g + (long long)al * N + rbeg;
    double2 s = make_double2(0, 0);
    for (int i0 = 0; i0 < nr; i0 += 16) {
      double2 gv[16];
#pragma unroll
      for (int u = 0; u < 16; ++u) gv[u] = (i0 + u < nr) ? __ldcg(gp + i0 + u) : make_double2(0, 0);
#pragma unroll
      for (int u = 0; u < 16; ++u)
        if (i0 + u < nr) s = cadd(s, cmul(P[(size_t)q * RS + i0 + u], gv[u]));
    }
    a.partVg[(size_t)blockIdx.x * BW * NGMAX + e] = s;
  }
  if (!sync_grid()) return;
  // Sum of the CTAs' partials in CTA order, the loads of 8 partials issued together
  auto sum_parts = [&](const double2* base, size_t stride, int e) {
    double2 s = make_double2(0, 0);
    for (int c0 = 0; c0 < G; c0 += 8) {
      double2 pv[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) pv[u] = (c0 + u < G) ? ldcg2(base + (size_t)(c0 + u) * stride + e) : make_double2(0, 0);
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (c0 + u < G) s = cadd(s, pv[u]);
    }
    return s;
  };
  // every CTA: y = V^T g (needed after the T factor; reduced while CTA 0 forms T)
  for (int e = tid; e < BW * a.ng; e += PQ_THREADS) s_y[e] = sum_parts(a.partVg, (size_t)BW * NGMAX, e);   // [q + al*BW]
  // T factor (ZLARFT forward columnwise): T[i][i] = tau_i, T[0:i, i] = -tau_i T[0:i, 0:i] G[0:i, i]
  if (blockIdx.x == 0) {
    for (int e = tid; e < BW * BW; e += PQ_THREADS) s_T[e] = sum_parts(a.partG, (size_t)BW * BW, e);   // G for now (qi + qj * BW)
    __syncthreads();
    // column by column on one warp; column i of T is built in s_w from G(:, i) before T(:, i) is
    // stored
    if (tid < BW) {
      for (int i = 0; i < BW; ++i) {
        s_w[tid] = (tid < i && i < nref) ? s_T[tid + i * BW] : make_double2(0, 0);
        __syncwarp();
        double2 t = make_double2(0, 0);
        if (i < nref && tid < i) {
          for (int l = tid; l < i; ++l) t = cadd(t, cmul(s_T[tid + l * BW], s_w[l]));   // T[tid][l] for l < i
          t = cscale(cmul(s_tau[i], t), -1.0);
        } else if (i < nref && tid == i) {
          t = s_tau[i];
        }
        // column i of the G storage is no longer needed below the diagonal: the T entries of
        // rows < i overwrite G(0:i, i); rows >= i become T's diagonal and zeros
        s_T[tid + i * BW] = t;
        __syncwarp();
      }
    }
    __syncthreads();
    // s_T now holds T upper triangular; G entries below the diagonal were overwritten with 0
    for (int e = tid; e < BW * BW; e += PQ_THREADS) a.Tout[e] = s_T[e];
  }
  if (!sync_grid()) return;
  // g <- g - conj(V) T^T (V^T g)
  for (int e = tid; e < BW * BW; e += PQ_THREADS) s_T[e] = ldcg2(a.Tout + e);
  __syncthreads();
  // z = T^T y into s_w-sized scratch: z[j][al] = sum_{i <= j} T[i][j] y[i][al]
  __shared__ double2 s_z[BW * NGMAX];
  for (int e = tid; e < BW * a.ng; e += PQ_THREADS) {
    const int j = e % BW, al = e / BW;
    double2 s = make_double2(0, 0);
    for (int i = 0; i <= j; ++i) s = cadd(s, cmul(s_T[i + j * BW], s_y[i + al * BW]));
    s_z[e] = s;
  }
  __syncthreads();
  for (int e = tid; e < nr * a.ng; e += PQ_THREADS) {
    const int i = e % nr, al = e / nr;
    double2 s = make_double2(0, 0);
    for (int q = 0; q < nref; ++q) s = cadd(s, cmul(cconj(vval(q, i)), s_z[q + al * BW]));
    double2* gp = a.g + (long long)al * N + rbeg + i;
    *gp = csub(*gp, s);
  }
}


// Diagonal 64 x 64 tiles of A22 made full Hermitian (lower stored, upper = conj of lower,
// diagonal real), column-major per tile: Dsym[I][c*64 + r].  Rows/columns past N are zero.
constexpr int SD_LD = 65;
constexpr size_t SD_SMEM = (size_t)64 * SD_LD * sizeof(double2);
__global__ void __launch_bounds__(256) k_symdiag(const double2* __restrict__ A, long long N, long long k0,
                                                 double2* __restrict__ Dsym) {
  // the tile's lower half read once with coalesced loads into sL [c][r], then written out full
  extern __shared__ __align__(16) double2 sL[];
  const long long I0 = k0 + (long long)blockIdx.x * 64;
  double2* D = Dsym + (size_t)blockIdx.x * 64 * 64;
  for (int e = threadIdx.x; e < 64 * 64; e += 256) {
    const int r = e & 63, c = e >> 6;
    const long long gr = I0 + r, gc = I0 + c;
    sL[c * SD_LD + r] = (r >= c && gr < N && gc < N) ? A[gr + gc * N] : make_double2(0, 0);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 64 * 64; e += 256) {
    const int r = e & 63, c = e >> 6;
    const long long gr = I0 + r, gc = I0 + c;
    double2 v = make_double2(0, 0);
    if (gr < N && gc < N) {
      if (r > c) v = sL[c * SD_LD + r];
      else if (r < c) v = cconj(sL[r * SD_LD + c]);
      else v = make_double2(sL[c * SD_LD + r].x, 0.0);
    }
    D[e] = v;
  }
}

// D += A B with A 16x16 (a_i: row gq + 8*(i%2), k = tq + 4*(i/2)) and B 16x8 (b_j: k = tq + 4*j,
// column gq): FP64 tensor-core MMA.
__device__ __forceinline__ void dmma16(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]), "d"(b[1]),
        "d"(b[2]), "d"(b[3]));
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
  const unsigned sh = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sh), "l"(src), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N_>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N_) : "memory"); }

// X = A22 V, A22 Hermitian (lower triangle of A from row/column k0), V = Vp (32 columns).
// CTA (I, s): the 64 rows I of X, column blocks J of A22 in split s, K staged in chunks of 32
// through a two-stage cp.async ring.  The A operand of chunk (J, kc) is A[I, J] (J < I, staged
// k-major), conj(A[J, I])^T (J > I, staged row-major, conjugated when the fragment is built) or
// the symmetrised diagonal tile (J = I).  Complex products as real MMAs with the real and
// imaginary parts concatenated along k: X_re = [Ar | Ai] [Vr; -Vi], X_im = [Ar | Ai] [Vi; Vr].
// Warp (wr, wc): rows 16 wr .. +16, columns 16 wc .. +16 (two 8-wide n blocks).
constexpr int HM_LDA = 66;   // sA[k][row], 64 rows + 2 (conflict-free fragment loads)
constexpr int HM_LDT = 36;   // sAT[row][k], 32 k + 4
constexpr int HM_LDV = 36;   // sV[col][k], 32 k + 4 (the staging writes along k and the fragment
                             // reads of 8 columns x 4 k both fall on distinct banks)
constexpr int HM_ABUF = 64 * HM_LDT;   // >= 32 * HM_LDA; union of the two A layouts
constexpr int HM_STAGE = HM_ABUF + 32 * HM_LDV;
constexpr size_t HM_SMEM = 2 * (size_t)HM_STAGE * sizeof(double2);

__global__ void __launch_bounds__(256, 2) k_hemm2(const double2* __restrict__ A, long long N, long long k0,
                                                  const double2* __restrict__ Dsym, const double2* __restrict__ V,
                                                  int nI, int chunkJ, double2* __restrict__ Xpart) {
  extern __shared__ __align__(16) double2 hs[];
  const int I = blockIdx.x, sp = blockIdx.y;
  const int J0 = sp * chunkJ, J1 = min(J0 + chunkJ, nI);
  const long long m = N - k0;
  const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  const int wr = wp & 3, wc = wp >> 2, gq = lane >> 2, tq = lane & 3;
  const long long rI = k0 + (long long)I * 64;

  double accr[2][4], acci[2][4];
#pragma unroll
  for (int nb = 0; nb < 2; ++nb)
#pragma unroll
    for (int k = 0; k < 4; ++k) accr[nb][k] = acci[nb][k] = 0.0;
  const int nch = 2 * max(0, J1 - J0);

  auto stage = [&](int c, int buf) {
    const int J = J0 + (c >> 1), kc = (c & 1) * 32;
    double2* sA = hs + (size_t)buf * HM_STAGE;
    double2* sV = sA + HM_ABUF;
    const long long cJ = k0 + (long long)J * 64 + kc;   // first global index of the k range
    if (J < I) {
      for (int e = tid; e < 64 * 32; e += 256) {
        const int r = e & 63, k = e >> 6;
        const long long gr = rI + r, gc = cJ + k;
        const bool ok = gr < N && gc < N;
        cp_async16(sA + k * HM_LDA + r, ok ? A + gr + gc * N : A, ok);
      }
    } else if (J > I) {
      for (int e = tid; e < 64 * 32; e += 256) {
        const int k = e & 31, r = e >> 5;
        const long long gr = cJ + k, gc = rI + r;   // stored element A[gr, gc], gr > gc
        const bool ok = gr < N && gc < N;
        cp_async16(sA + r * HM_LDT + k, ok ? A + gr + gc * N : A, ok);
      }
    } else {
      const double2* D = Dsym + (size_t)I * 64 * 64;
      for (int e = tid; e < 64 * 32; e += 256) {
        const int r = e & 63, k = e >> 6;
        cp_async16(sA + k * HM_LDA + r, D + (size_t)(kc + k) * 64 + r, true);
      }
    }
    for (int e = tid; e < 32 * 32; e += 256) {
      const int k = e & 31, col = e >> 5;
      const long long gr = cJ + k;
      const bool ok = gr < N;
      cp_async16(sV + col * HM_LDV + k, ok ? V + gr + (long long)col * N : V, ok);
    }
    cp_async_commit();
  };

  if (nch > 0) stage(0, 0);
  if (nch > 1) stage(1, 1);
  for (int c = 0; c < nch; ++c) {
    if (c + 1 < nch) cp_async_wait<1>();
    else cp_async_wait<0>();
    __syncthreads();
    const double2* sA = hs + (size_t)(c & 1) * HM_STAGE;
    const double2* sV = sA + HM_ABUF;
    const bool tr = (J0 + (c >> 1)) > I;
    const int r0 = wr * 16 + gq, r1 = r0 + 8;
#pragma unroll
    for (int kk = 0; kk < 32; kk += 8) {
      const int ka = kk + tq, kb = ka + 4;
      double2 x00, x10, x01, x11;
      if (tr) {
        x00 = cconj(sA[r0 * HM_LDT + ka]);
        x10 = cconj(sA[r1 * HM_LDT + ka]);
        x01 = cconj(sA[r0 * HM_LDT + kb]);
        x11 = cconj(sA[r1 * HM_LDT + kb]);
      } else {
        x00 = sA[ka * HM_LDA + r0];
        x10 = sA[ka * HM_LDA + r1];
        x01 = sA[kb * HM_LDA + r0];
        x11 = sA[kb * HM_LDA + r1];
      }
      const double a[8] = {x00.x, x10.x, x01.x, x11.x, x00.y, x10.y, x01.y, x11.y};
#pragma unroll
      for (int nb = 0; nb < 2; ++nb) {
        const int col = wc * 16 + nb * 8 + gq;
        const double2 v0 = sV[col * HM_LDV + ka], v1 = sV[col * HM_LDV + kb];
        const double bre[4] = {v0.x, v1.x, -v0.y, -v1.y};
        const double bim[4] = {v0.y, v1.y, v0.x, v1.x};
        dmma16(accr[nb], a, bre);
        dmma16(acci[nb], a, bim);
      }
    }
    __syncthreads();
    if (c + 2 < nch) stage(c + 2, c & 1);
  }
#pragma unroll
  for (int nb = 0; nb < 2; ++nb)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const long long row = rI + wr * 16 + gq + ((k >> 1) ? 8 : 0);
      const int col = wc * 16 + nb * 8 + 2 * tq + (k & 1);
      if (row < N) Xpart[((size_t)sp * 32 + col) * (size_t)m + (size_t)(row - k0)] = make_double2(accr[nb][k], acci[nb][k]);
    }
}

constexpr int XR_LD = 65;   // row stride of sX, sV: odd, so the Gram loads of 32 columns hit distinct banks
constexpr size_t XR_SMEM = (size_t)(32 * XR_LD + 32 * 32 + 32 * XR_LD) * sizeof(double2);
// X = sum of the split partials; Y = X T into Wp; partial G_b = V_b^H Y_b over the 64 rows of
// this block (Gpart[b][i + 32 j]).  Every sum keeps its order; the independent sums of a thread
// are interleaved and the split partials' loads issued together (the kernel is latency-bound).
__global__ void __launch_bounds__(256) k_xreduce(const double2* __restrict__ Xpart, int S, long long N, long long k0,
                                                 const double2* __restrict__ T, const double2* __restrict__ V,
                                                 double2* __restrict__ Wp, double2* __restrict__ Gpart) {
  extern __shared__ __align__(16) double2 xsm[];   // sX [32][XR_LD], sT [32][32], sV [32][XR_LD]
  double2* sX = xsm;
  double2* sT = sX + 32 * XR_LD;
  double2* sV = sT + 32 * 32;
  const long long m = N - k0;
  const long long rb = (long long)blockIdx.x * 64;
  const int tid = threadIdx.x;
  for (int e = tid; e < 32 * 32; e += 256) sT[e] = T[e];
  for (int e = tid; e < 32 * 64; e += 256) {
    const int r = e & 63, c = e >> 6;
    const long long rr = rb + r;
    double2 x = make_double2(0, 0), v = make_double2(0, 0);
    if (rr < m) {
      double2 xp[8];
#pragma unroll
      for (int s = 0; s < 8; ++s) xp[s] = (s < S) ? Xpart[((size_t)s * 32 + c) * (size_t)m + rr] : make_double2(0, 0);
#pragma unroll
      for (int s = 0; s < 8; ++s)
        if (s < S) x = cadd(x, xp[s]);
      v = V[k0 + rr + (long long)c * N];
    }
    sX[c * XR_LD + r] = x;
    sV[c * XR_LD + r] = v;
  }
  __syncthreads();
  // y[u] = sum_{i <= j_u} X[r][i] T[i][j_u], j_u = tid/64 + 4u, the eight chains interleaved
  double2 y[8];
  const int r = tid & 63, jb0 = tid >> 6;
#pragma unroll
  for (int u = 0; u < 8; ++u) y[u] = make_double2(0, 0);
  for (int i = 0; i <= jb0 + 28; ++i) {
    const double2 xi = sX[i * XR_LD + r];
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (i <= jb0 + 4 * u) y[u] = cadd(y[u], cmul(xi, sT[i + (jb0 + 4 * u) * 32]));
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int j = jb0 + 4 * u;
    sX[j * XR_LD + r] = y[u];
    if (rb + r < m) Wp[k0 + rb + r + (long long)j * N] = y[u];
  }
  __syncthreads();
  // G[i][j] = sum_r conj(V[r][i]) Y[r][j]: thread t takes (i, j) = (t mod 32, t/32 + 8k), k < 4
  {
    const int i = tid & 31, j0 = tid >> 5;
    double2 g4[4] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    for (int rr = 0; rr < 64; ++rr) {
      const double2 vi = sV[i * XR_LD + rr];
#pragma unroll
      for (int k = 0; k < 4; ++k) g4[k] = cadd(g4[k], cmulc(vi, sX[(j0 + 8 * k) * XR_LD + rr]));
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) Gpart[(size_t)blockIdx.x * 1024 + i + 32 * (j0 + 8 * k)] = g4[k];
  }
}

// M = T^H G, G = sum of the block partials (one CTA, fixed summation order)
__global__ void __launch_bounds__(1024) k_mform(const double2* __restrict__ Gpart, int nb, const double2* __restrict__ T,
                                                double2* __restrict__ M) {
  __shared__ double2 sG[1024];
  __shared__ double2 sT[1024];
  const int e = threadIdx.x;
  double2 t = make_double2(0, 0);
  for (int b0 = 0; b0 < nb; b0 += 8) {   // in block order, 8 loads issued together
    double2 pv[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) pv[u] = (b0 + u < nb) ? __ldcg(Gpart + (size_t)(b0 + u) * 1024 + e) : make_double2(0, 0);
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (b0 + u < nb) t = cadd(t, pv[u]);
  }
  sG[e] = t;
  sT[e] = T[e];
  __syncthreads();
  const int i = e & 31, j = e >> 5;
  double2 s = make_double2(0, 0);
  for (int l = 0; l <= i; ++l) s = cadd(s, cmulc(sT[l + i * 32], sG[l + j * 32]));   // conj(T[l][i]) G[l][j]
  M[i + 32 * j] = s;
}

// W = Y - 1/2 V M (in place in Wp, rows k0..N-1): 32 rows per CTA, V staged column by column
// with coalesced loads; element (r, j) sums i in order as before
constexpr int WF_LD = 33;
__global__ void __launch_bounds__(256) k_wform(long long N, long long k0, const double2* __restrict__ V,
                                               const double2* __restrict__ M, double2* __restrict__ Wp) {
  __shared__ double2 sM[1024];
  __shared__ double2 sVb[32 * WF_LD];
  const int tid = threadIdx.x;
  const long long r0 = k0 + (long long)blockIdx.x * 32;
  for (int e = tid; e < 1024; e += 256) sM[e] = M[e];
  for (int e = tid; e < 32 * 32; e += 256) {
    const int rr = e & 31, i = e >> 5;
    sVb[i * WF_LD + rr] = (r0 + rr < N) ? V[r0 + rr + (long long)i * N] : make_double2(0, 0);
  }
  __syncthreads();
  const int rr = tid & 31, jg = tid >> 5;   // columns j = jg + 8u, u < 4
  if (r0 + rr >= N) return;
  double2 t[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) t[u] = make_double2(0, 0);
  for (int i = 0; i < 32; ++i) {
    const double2 vi = sVb[i * WF_LD + rr];
#pragma unroll
    for (int u = 0; u < 4; ++u) t[u] = cadd(t[u], cmul(vi, sM[i + 32 * (jg + 8 * u)]));
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    double2* w = Wp + r0 + rr + (long long)(jg + 8 * u) * N;
    *w = csub(*w, cscale(t[u], 0.5));
  }
}


// Look-ahead group of panels.  Vacc, Wacc hold the group's V and W side by side (32 columns per
// panel, leading dimension N); K = 32 * (panels already factored in the group).

// Strip of the next panel: columns c in [c0, c0+32), rows r >= c, get the pending updates of the
// group's earlier panels, A[r,c] -= sum_{q<K} V[r,q] conj(W[c,q]) + W[r,q] conj(V[c,q]).
// One warp per row (lane = column); the column rows of V and W in shared memory.
__global__ void __launch_bounds__(256) k_strip_update(double2* __restrict__ A, long long N, long long c0, int K,
                                                      const double2* __restrict__ V, const double2* __restrict__ W) {
  // sVc, sWc [K][32]: the strip's column rows; sVr, sWr [K][33]: this CTA's 32 rows (coalesced
  // loads); thread (lane = row, warp w) takes the columns w + 8v; sums in the order as before
  extern __shared__ __align__(16) double2 ssm[];
  double2* sVc = ssm;
  double2* sWc = ssm + (size_t)K * 32;
  double2* sVr = sWc + (size_t)K * 32;
  double2* sWr = sVr + (size_t)K * 33;
  const long long rb = c0 + (long long)blockIdx.x * 32;
  for (int e = threadIdx.x; e < K * 32; e += 256) {
    const int q = e >> 5, c = e & 31;
    const long long rc = c0 + c, rr = rb + c;
    sVc[e] = rc < N ? V[rc + (long long)q * N] : make_double2(0, 0);
    sWc[e] = rc < N ? W[rc + (long long)q * N] : make_double2(0, 0);
    sVr[q * 33 + c] = rr < N ? V[rr + (long long)q * N] : make_double2(0, 0);
    sWr[q * 33 + c] = rr < N ? W[rr + (long long)q * N] : make_double2(0, 0);
  }
  __syncthreads();
  const int u = threadIdx.x & 31, cg = threadIdx.x >> 5;
  const long long r = rb + u;
  if (r >= N) return;
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const int c = cg + 8 * v;
    if (c0 + c >= N || r < c0 + c) continue;
    double2 t0 = make_double2(0, 0), t1 = t0;
    for (int q = 0; q < K; q += 2) {
      t0 = cadd(t0, cadd(cmulc(sWc[q * 32 + c], sVr[q * 33 + u]), cmulc(sVc[q * 32 + c], sWr[q * 33 + u])));
      t1 = cadd(t1, cadd(cmulc(sWc[(q + 1) * 32 + c], sVr[(q + 1) * 33 + u]),
                         cmulc(sVc[(q + 1) * 32 + c], sWr[(q + 1) * 33 + u])));
    }
    const long long idx = r + (c0 + c) * N;
    double2 a = csub(A[idx], cadd(t0, t1));
    if (r == c0 + c) a.y = 0.0;
    A[idx] = a;
  }
}

// Correction Gram matrices over 64-row blocks from row k1: which = 0: C1 = Wacc^H V2,
// which = 1: C2 = Vacc^H V2 (K x 32 each, part[b][which][i + K j]).  Rows staged in shared memory.
constexpr int CP_LD = 65;
__global__ void __launch_bounds__(256) k_cpart(long long N, long long k1, int K, const double2* __restrict__ Vacc,
                                               const double2* __restrict__ Wacc, const double2* __restrict__ V2,
                                               double2* __restrict__ part) {
  // sL [K][CP_LD], sV [32][CP_LD]: the odd row stride keeps a warp's K different rows of sL on
  // distinct banks
  extern __shared__ __align__(16) double2 csm[];
  const int which = blockIdx.y;
  const double2* L = which ? Vacc : Wacc;
  double2* sL = csm;
  double2* sV = csm + (size_t)K * CP_LD;
  const long long rb = k1 + (long long)blockIdx.x * 64;
  for (int e = threadIdx.x; e < K * 64; e += 256) {
    const int u = e & 63, i = e >> 6;
    const long long r = rb + u;
    sL[i * CP_LD + u] = r < N ? L[r + (long long)i * N] : make_double2(0, 0);
  }
  for (int e = threadIdx.x; e < 32 * 64; e += 256) {
    const int u = e & 63, j = e >> 6;
    const long long r = rb + u;
    sV[j * CP_LD + u] = r < N ? V2[r + (long long)j * N] : make_double2(0, 0);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < K * 32; e += 256) {
    const int i = e % K, j = e / K;
    double2 t0 = make_double2(0, 0), t1 = t0;
    for (int u = 0; u < 64; u += 2) {
      t0 = cadd(t0, cmulc(sL[i * CP_LD + u], sV[j * CP_LD + u]));
      t1 = cadd(t1, cmulc(sL[i * CP_LD + u + 1], sV[j * CP_LD + u + 1]));
    }
    part[((size_t)blockIdx.x * 2 + which) * K * 32 + e] = cadd(t0, t1);
  }
}
// C12[which][i + K j] = sum over the blocks (fixed order); grid over entries
__global__ void __launch_bounds__(256) k_creduce(const double2* __restrict__ part, int nb, int K, double2* __restrict__ C12) {
  const int e = blockIdx.x * 256 + threadIdx.x;
  if (e >= 2 * K * 32) return;
  double2 t0 = make_double2(0, 0), t1 = t0;
  int b = 0;
  for (; b + 1 < nb; b += 2) {
    t0 = cadd(t0, part[(size_t)b * 2 * K * 32 + e]);
    t1 = cadd(t1, part[(size_t)(b + 1) * 2 * K * 32 + e]);
  }
  if (b < nb) t0 = cadd(t0, part[(size_t)b * 2 * K * 32 + e]);
  C12[e] = cadd(t0, t1);
}
// X (the first split partial, [32][m]) -= Vacc C1 + Wacc C2 for the rows from k1: one warp per
// row, lane = column; C1, C2 in shared memory.
__global__ void __launch_bounds__(256) k_xcorr(double2* __restrict__ X0, long long N, long long k1, int K,
                                               const double2* __restrict__ Vacc, const double2* __restrict__ Wacc,
                                               const double2* __restrict__ C12) {
  // C1 [K][32] (i + K j), C2, then the 32 rows of Vacc and Wacc [K][33] (staged with coalesced
  // loads); element (rr, c) sums i in order as before, 32 rows per CTA, lanes along the rows
  extern __shared__ __align__(16) double2 xsm2[];
  double2* sVa = xsm2 + 2 * K * 32;
  double2* sWa = sVa + (size_t)K * 33;
  const long long m = N - k1;
  const long long rr0 = (long long)blockIdx.x * 32;
  for (int e = threadIdx.x; e < 2 * K * 32; e += 256) xsm2[e] = C12[e];
  for (int e = threadIdx.x; e < K * 32; e += 256) {
    const int u = e & 31, i = e >> 5;
    const bool ok = rr0 + u < m;
    sVa[i * 33 + u] = ok ? Vacc[k1 + rr0 + u + (long long)i * N] : make_double2(0, 0);
    sWa[i * 33 + u] = ok ? Wacc[k1 + rr0 + u + (long long)i * N] : make_double2(0, 0);
  }
  __syncthreads();
  const int u = threadIdx.x & 31, cg = threadIdx.x >> 5;   // columns c = cg + 8v, v < 4
  const long long rr = rr0 + u;
  if (rr >= m) return;
  double2 t0[4], t1[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) t0[v] = t1[v] = make_double2(0, 0);
  for (int i = 0; i < K; ++i) {
    const double2 va = sVa[i * 33 + u], wa = sWa[i * 33 + u];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int c = cg + 8 * v;
      t0[v] = cadd(t0[v], cmul(va, xsm2[i + K * c]));
      t1[v] = cadd(t1[v], cmul(wa, xsm2[K * 32 + i + K * c]));
    }
  }
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const int c = cg + 8 * v;
    X0[(size_t)c * m + rr] = csub(X0[(size_t)c * m + rr], cadd(t0[v], t1[v]));
  }
}

// ----------------------------------------------------------------------------- stage 2
// Band storage: column j holds A[j + o, j] for o = 0 .. LDB-1 (the band, o <= b, and room for
// the bulges, o <= 2b - 1).
constexpr int LDB = 2 * BW + 2;
constexpr int BG_WARPS = 4;                 // sweep workers per CTA
constexpr int BG_LD = BW + 1;               // padded row length of the per-warp work tiles
constexpr int BG_WARP_TILE = 3 * BW * BG_LD + 2 * BW;   // Bs, Ds, B1s, v, w (double2) per warp

__device__ __forceinline__ long long nsteps_of(long long N, long long s) { return (N - 1 - s + BW - 1) / BW; }
// sum_{u=1}^{U} ceil(u / b)
__device__ __host__ __forceinline__ long long ceil_sum(long long U) {
  if (U <= 0) return 0;
  const long long q = U / BW, r = U % BW;
  return BW * q * (q + 1) / 2 + r * (q + 1);
}
// index of the first reflector of sweep s in the flat tau2 array
__device__ __host__ __forceinline__ long long tau2_offset(long long N, long long s) {
  return ceil_sum(N - 1) - ceil_sum(N - 1 - s);
}

__global__ void __launch_bounds__(256) k_band_extract(const double2* __restrict__ A, long long N, double2* __restrict__ AB) {
  const long long j = blockIdx.x;
  for (int o = threadIdx.x; o < LDB; o += blockDim.x) {
    double2 v = make_double2(0, 0);
    if (o <= BW && j + o < N) v = A[(j + o) + j * N];
    if (o == 0) v.y = 0.0;
    AB[j * LDB + o] = v;
  }
}

struct BulgeArgs {
  double2* AB;
  long long N;
  double2* A;            // upper triangle: reflector vectors (sweep s in column N-1-s, rows 0..)
  double2* tau2;         // [tau2_offset(N, s) + t]
  double2* g;            // [ng][N]
  int ng;
  unsigned int* prog;    // [N] steps published per sweep
  int* err;
  int store;             // keep the reflectors for the eigenvector back-transform
  int nprob;             // independent bands chased in one launch (eigenvalues only when > 1)
  long long ab_stride;   // elements between consecutive bands in AB
  long long prog_stride; // entries between consecutive progress arrays
};

// One step of sweep s (warp-wide; lane i <-> row r0 + i of the step's blocks).  All the
// blocks the step reads (bulge block B_t, diagonal block D_t, block below B_{t+1}) are fetched
// at once with cp.async into the warp's shared tiles, so the step pays one L2 round trip; the
// dot products run with four independent partial sums per lane.
__device__ __forceinline__ void cpa16(double2* dst, const double2* src, bool valid) {
  const unsigned sh = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sh), "l"(src), "r"(valid ? 16 : 0) : "memory");
}

__device__ void bulge_step(const BulgeArgs& a, long long s, long long t, double2* Bs, double2* Ds, double2* B1s,
                           double2* vs, double2* ws) {
  const int lane = threadIdx.x & 31;
  const long long N = a.N;
  double2* AB = a.AB;
  const long long r0 = s + 1 + t * BW;
  const int L = (int)min((long long)BW, N - r0);
  const long long c0 = r0 - BW;   // first column of the bulge block (t >= 1)
  const long long r1 = r0 + L;
  const int L1 = (r1 < N) ? (int)min((long long)BW, N - r1) : 0;
  // ---- fetch
  if (t > 0) {
#pragma unroll 8
    for (int q = 0; q < BW; ++q) cpa16(Bs + lane * BG_LD + q, AB + (c0 + q) * LDB + (BW + lane - q), lane < L);
  }
  for (int q = 0; q < L; ++q) {
    const bool ok = lane >= q && lane < L;
    cpa16(Ds + lane * BG_LD + q, ok ? AB + (r0 + q) * LDB + (lane - q) : AB, ok);
  }
  for (int q = 0; q < L; ++q) cpa16(B1s + lane * BG_LD + q, AB + (r0 + q) * LDB + (L + lane - q), lane < L1);
  asm volatile("cp.async.commit_group;" ::: "memory");
  double2 gv[NGMAX];
#pragma unroll
  for (int al2 = 0; al2 < NGMAX; ++al2)
    gv[al2] = (al2 < a.ng && lane < L) ? __ldcg(a.g + (long long)al2 * N + r0 + lane) : make_double2(0, 0);
  double2 x = make_double2(0, 0);
  if (t == 0 && lane < L) x = __ldcg(AB + s * LDB + 1 + lane);
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncwarp();
  if (t > 0) x = Bs[lane * BG_LD];
  // ---- reflector (ZLARFG)
  double xn2 = (lane >= 1 && lane < L) ? x.x * x.x + x.y * x.y : 0.0;
  xn2 = warp_sum(xn2);
  const double2 al = make_double2(__shfl_sync(0xffffffffu, x.x, 0), __shfl_sync(0xffffffffu, x.y, 0));
  double2 tau, scal;
  double beta;
  if (xn2 == 0.0 && al.y == 0.0) {
    tau = make_double2(0, 0);
    scal = make_double2(0, 0);
    beta = al.x;
  } else {
    beta = -copysign(sqrt(al.x * al.x + al.y * al.y + xn2), al.x);
    tau = make_double2((beta - al.x) / beta, -al.y / beta);
    const double2 den = make_double2(al.x - beta, al.y);
    const double dd = den.x * den.x + den.y * den.y;
    scal = make_double2(den.x / dd, -den.y / dd);
  }
  const double2 v = (lane == 0) ? make_double2(1.0, 0.0) : (lane < L ? cmul(x, scal) : make_double2(0, 0));
  vs[lane] = v;
  // Hermitian fill of D (upper = conj of lower, real diagonal)
  if (lane < L)
    for (int q = 0; q <= lane; ++q) {
      double2 d = Ds[lane * BG_LD + q];
      if (q == lane) {
        d.y = 0.0;
        Ds[lane * BG_LD + q] = d;
      } else {
        Ds[q * BG_LD + lane] = cconj(d);
      }
    }
  __syncwarp();
  // ---- annihilated column and the left application to the rest of the bulge block
  if (lane < L) {
    const double2 nv = (lane == 0) ? make_double2(beta, 0.0) : make_double2(0, 0);
    if (t == 0) AB[s * LDB + 1 + lane] = nv;
    else AB[c0 * LDB + BW + lane] = nv;
  }
  if (t > 0) {
    if (lane >= 1) {   // w_q = sum_i conj(v_i) B(i, q), lane q
      double2 w0 = make_double2(0, 0), w1 = w0, w2 = w0, w3 = w0;
      for (int i = 0; i < L; i += 4) {
        w0 = cadd(w0, cmulc(vs[i], Bs[i * BG_LD + lane]));
        if (i + 1 < L) w1 = cadd(w1, cmulc(vs[i + 1], Bs[(i + 1) * BG_LD + lane]));
        if (i + 2 < L) w2 = cadd(w2, cmulc(vs[i + 2], Bs[(i + 2) * BG_LD + lane]));
        if (i + 3 < L) w3 = cadd(w3, cmulc(vs[i + 3], Bs[(i + 3) * BG_LD + lane]));
      }
      ws[lane] = cadd(cadd(w0, w1), cadd(w2, w3));
    }
    __syncwarp();
    if (lane < L) {
      const double2 cv = cmul(cconj(tau), v);
#pragma unroll 4
      for (int q = 1; q < BW; ++q)
        AB[(c0 + q) * LDB + (BW + lane - q)] = csub(Bs[lane * BG_LD + q], cmul(cv, ws[q]));
    }
    __syncwarp();
  }
  // ---- two-sided update of D: D <- H^H D H
  double2 y = make_double2(0, 0);
  if (lane < L) {
    double2 y1 = y, y2 = y, y3 = y;
    for (int q = 0; q < L; q += 4) {
      y = cadd(y, cmul(Ds[lane * BG_LD + q], vs[q]));
      if (q + 1 < L) y1 = cadd(y1, cmul(Ds[lane * BG_LD + q + 1], vs[q + 1]));
      if (q + 2 < L) y2 = cadd(y2, cmul(Ds[lane * BG_LD + q + 2], vs[q + 2]));
      if (q + 3 < L) y3 = cadd(y3, cmul(Ds[lane * BG_LD + q + 3], vs[q + 3]));
    }
    y = cadd(cadd(y, y1), cadd(y2, y3));
  }
  // v^H y (real for Hermitian D) and, interleaved, v^T g of the velocity vectors
  double pvx = cmulc(v, y).x;
  double2 sg[NGMAX];
#pragma unroll
  for (int al2 = 0; al2 < NGMAX; ++al2) sg[al2] = cmul(v, gv[al2]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    pvx += __shfl_xor_sync(0xffffffffu, pvx, o);
#pragma unroll
    for (int al2 = 0; al2 < NGMAX; ++al2) {
      if (al2 < a.ng) {
        sg[al2].x += __shfl_xor_sync(0xffffffffu, sg[al2].x, o);
        sg[al2].y += __shfl_xor_sync(0xffffffffu, sg[al2].y, o);
      }
    }
  }
  const double t2 = tau.x * tau.x + tau.y * tau.y;
  const double2 w = csub(cmul(tau, y), cscale(v, 0.5 * t2 * pvx));
  ws[lane] = w;
  __syncwarp();
  if (lane < L)
#pragma unroll 4
    for (int q = 0; q <= lane; ++q) {
      double2 d = csub(Ds[lane * BG_LD + q], cadd(cmulc(ws[q], v), cmulc(vs[q], w)));   // v_i conj(w_q) + w_i conj(v_q)
      if (q == lane) d.y = 0.0;
      AB[(r0 + q) * LDB + (lane - q)] = d;
    }
  // ---- right application to the block below: B1 <- B1 H
  if (L1 > 0) {
    double2 z = make_double2(0, 0);
    if (lane < L1) {
      double2 z1 = z, z2 = z, z3 = z;
      for (int q = 0; q < L; q += 4) {
        z = cadd(z, cmul(B1s[lane * BG_LD + q], vs[q]));
        if (q + 1 < L) z1 = cadd(z1, cmul(B1s[lane * BG_LD + q + 1], vs[q + 1]));
        if (q + 2 < L) z2 = cadd(z2, cmul(B1s[lane * BG_LD + q + 2], vs[q + 2]));
        if (q + 3 < L) z3 = cadd(z3, cmul(B1s[lane * BG_LD + q + 3], vs[q + 3]));
      }
      z = cadd(cadd(z, z1), cadd(z2, z3));
      const double2 tz = cmul(tau, z);
#pragma unroll 4
      for (int q = 0; q < L; ++q)
        AB[(r0 + q) * LDB + (L + lane - q)] = csub(B1s[lane * BG_LD + q], cmul(tz, cconj(vs[q])));
    }
  }
  // ---- velocity vectors: g <- g - tau conj(v) (v^T g)
  if (lane < L) {
    const double2 tcv = cmul(tau, cconj(v));
#pragma unroll
    for (int al2 = 0; al2 < NGMAX; ++al2)
      if (al2 < a.ng) a.g[(long long)al2 * N + r0 + lane] = csub(gv[al2], cmul(tcv, sg[al2]));
  }
  if (a.store) {
    if (lane < L) a.A[(r0 + lane - s - 1) + (N - 1 - s) * N] = v;
    if (lane == 0) a.tau2[tau2_offset(N, s) + t] = tau;
  }
  __syncwarp();
}

// Persistent bulge chasing: warp w of the grid runs sweeps w, w + W, w + 2W, ...; sweep s
// starts step t after sweep s-1 has published step t+2 (or finished): the elements of step t
// of sweep s have rows and columns <= s + 1 + (t+2) b, those of step t+3 of sweep s-1 rows
// >= s + (t+3) b + 1, so the two never touch the same element (nor the same rows of g).
__global__ void __launch_bounds__(32 * BG_WARPS, 1) k_bulge(BulgeArgs a) {
  extern __shared__ __align__(16) double2 bsm[];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2* Bs = bsm + (size_t)wid * BG_WARP_TILE;
  double2* Ds = Bs + BW * BG_LD;
  double2* B1s = Ds + BW * BG_LD;
  double2* vs = B1s + BW * BG_LD;
  double2* ws = vs + BW;
  const long long W = (long long)gridDim.x * BG_WARPS;
  const long long N = a.N;
  const long long np = a.nprob;
  // sweep u of the launch = sweep s = u / np of band q = u % np: sweeps are taken in increasing
  // u, and a sweep waits only on sweep s-1 of its own band (index u - np), so every wait is on a
  // sweep that some resident warp has already started or finished
  for (long long u = (long long)blockIdx.x * BG_WARPS + wid; u < np * (N - 1); u += W) {
    const long long q = u % np, s = u / np;
    BulgeArgs b = a;
    b.AB = a.AB + q * a.ab_stride;
    unsigned int* prog = a.prog + q * a.prog_stride;
    const long long ns = nsteps_of(N, s);
    const long long nprev = (s > 0) ? nsteps_of(N, s - 1) : 0;
    for (long long t = 0; t < ns; ++t) {
      if (s > 0) {
        const unsigned int need = (unsigned int)min(t + 3, nprev);
        int bad = 0;
        if (lane == 0) bad = wait_at_least(prog + s - 1, need, a.err) ? 0 : 1;
        bad = __shfl_sync(0xffffffffu, bad, 0);
        if (bad) return;
      }
      bulge_step(b, s, t, Bs, Ds, B1s, vs, ws);
      // publish: the warp barrier orders the lanes' writes before lane 0's release store
      __syncwarp();
      if (lane == 0) st_release(prog + s, (unsigned int)(t + 1));
    }
  }
}

// Stage 2 with one CTA of four warps per sweep.  After the fetch (all 128 threads) warp 0
// forms the reflector while warp 2 completes the Hermitian diagonal block; then the four updates,
// which need only v and tau, run concurrently: warp 0 the annihilated column, the velocity
// vectors and the stored reflector, warp 1 the left application to the bulge block, warp 2 the
// two-sided update of the diagonal block, warp 3 the right application to the block below.
constexpr int B4_THREADS = 128;
constexpr int B4_TILE = 3 * BW * BG_LD + 4 * BW + 8;   // Bs, Ds, B1s, v, w1, w2, scalars (double2)
constexpr size_t B4_SMEM = (size_t)B4_TILE * 16;

// Bs, Ds, B1s: the bulge block, the diagonal block and the block below; gv: warp 0's rows of the
// velocity vectors.  With pre, the previous step of the sweep has already placed them (Bs is its
// block below, updated in place; Ds, B1s and gv prefetched) except the corner of B1s, which the
// predecessor sweep's step t + 3 writes and which is read here after the wait.
__device__ void bulge_step4(const BulgeArgs& a, long long s, long long t, double2* Bs, double2* Ds, double2* B1s,
                            double2* tail, double2 (&gv)[NGMAX], bool pre) {
  double2* vs = tail;
  double2* w1 = vs + BW;
  double2* w2 = w1 + BW;
  double2* sc = w2 + BW;   // [0] tau, [1] (beta, 0)
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const long long N = a.N;
  double2* AB = a.AB;
  const long long r0 = s + 1 + t * BW;
  const int L = (int)min((long long)BW, N - r0);
  const long long c0 = r0 - BW;
  const long long r1 = r0 + L;
  const int L1 = (r1 < N) ? (int)min((long long)BW, N - r1) : 0;
  // ---- fetch (element e of each tile: row e % 32, column e / 32)
  if (!pre) {
    if (t > 0)
      for (int e = tid; e < BW * BW; e += B4_THREADS) {
        const int i = e & 31, q = e >> 5;
        cpa16(Bs + i * BG_LD + q, AB + (c0 + q) * LDB + (BW + i - q), i < L);
      }
    for (int e = tid; e < BW * BW; e += B4_THREADS) {
      const int i = e & 31, q = e >> 5;
      if (q < L) {
        const bool ok = i >= q && i < L;
        cpa16(Ds + i * BG_LD + q, ok ? AB + (r0 + q) * LDB + (i - q) : AB, ok);
        cpa16(B1s + i * BG_LD + q, AB + (r0 + q) * LDB + (L + i - q), i < L1);
      }
    }
  } else if (tid == 0 && L == BW && L1 == BW) {
    cpa16(B1s + (BW - 1) * BG_LD + (BW - 1), AB + (r0 + BW - 1) * LDB + L, true);
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
  if (wid == 0 && !pre) {
#pragma unroll
    for (int al2 = 0; al2 < NGMAX; ++al2)
      gv[al2] = (al2 < a.ng && lane < L) ? __ldcg(a.g + (long long)al2 * N + r0 + lane) : make_double2(0, 0);
  }
  double2 x = make_double2(0, 0);
  if (wid == 0 && t == 0 && lane < L) x = __ldcg(AB + s * LDB + 1 + lane);
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();
  // ---- reflector (warp 0) | Hermitian fill of D (warp 2)
  if (wid == 0) {
    if (t > 0) x = Bs[lane * BG_LD];
    double xn2 = (lane >= 1 && lane < L) ? x.x * x.x + x.y * x.y : 0.0;
    xn2 = warp_sum(xn2);
    const double2 al = make_double2(__shfl_sync(0xffffffffu, x.x, 0), __shfl_sync(0xffffffffu, x.y, 0));
    double2 tau, scal;
    double beta;
    if (xn2 == 0.0 && al.y == 0.0) {
      tau = make_double2(0, 0);
      scal = make_double2(0, 0);
      beta = al.x;
    } else {
      beta = -copysign(sqrt(al.x * al.x + al.y * al.y + xn2), al.x);
      tau = make_double2((beta - al.x) / beta, -al.y / beta);
      const double2 den = make_double2(al.x - beta, al.y);
      const double dd = den.x * den.x + den.y * den.y;
      scal = make_double2(den.x / dd, -den.y / dd);
    }
    vs[lane] = (lane == 0) ? make_double2(1.0, 0.0) : (lane < L ? cmul(x, scal) : make_double2(0, 0));
    if (lane == 0) {
      sc[0] = tau;
      sc[1] = make_double2(beta, 0.0);
    }
  } else if (wid == 2 && lane < L) {
    for (int q = 0; q <= lane; ++q) {
      double2 d = Ds[lane * BG_LD + q];
      if (q == lane) {
        d.y = 0.0;
        Ds[lane * BG_LD + q] = d;
      } else {
        Ds[q * BG_LD + lane] = cconj(d);
      }
    }
  }
  __syncthreads();
  const double2 tau = sc[0];
  const double2 v = vs[lane];
  if (wid == 0) {
    // annihilated column, velocity vectors, stored reflector
    if (lane < L) {
      const double2 nv = (lane == 0) ? sc[1] : make_double2(0, 0);
      if (t == 0) AB[s * LDB + 1 + lane] = nv;
      else AB[c0 * LDB + BW + lane] = nv;
    }
    double2 sg[NGMAX];
#pragma unroll
    for (int al2 = 0; al2 < NGMAX; ++al2) sg[al2] = cmul(v, gv[al2]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int al2 = 0; al2 < NGMAX; ++al2)
        if (al2 < a.ng) {
          sg[al2].x += __shfl_xor_sync(0xffffffffu, sg[al2].x, o);
          sg[al2].y += __shfl_xor_sync(0xffffffffu, sg[al2].y, o);
        }
    if (lane < L) {
      const double2 tcv = cmul(tau, cconj(v));
#pragma unroll
      for (int al2 = 0; al2 < NGMAX; ++al2)
        if (al2 < a.ng) a.g[(long long)al2 * N + r0 + lane] = csub(gv[al2], cmul(tcv, sg[al2]));
      if (a.store) a.A[(r0 + lane - s - 1) + (N - 1 - s) * N] = v;
    }
    if (a.store && lane == 0) a.tau2[tau2_offset(N, s) + t] = tau;
  } else if (wid == 1) {
    // left application to the bulge block: B <- H^H B (columns 1..31)
    if (t > 0) {
      if (lane >= 1) {
        double2 a0 = make_double2(0, 0), a1 = a0, a2 = a0, a3 = a0;
        for (int i = 0; i < L; i += 4) {
          a0 = cadd(a0, cmulc(vs[i], Bs[i * BG_LD + lane]));
          if (i + 1 < L) a1 = cadd(a1, cmulc(vs[i + 1], Bs[(i + 1) * BG_LD + lane]));
          if (i + 2 < L) a2 = cadd(a2, cmulc(vs[i + 2], Bs[(i + 2) * BG_LD + lane]));
          if (i + 3 < L) a3 = cadd(a3, cmulc(vs[i + 3], Bs[(i + 3) * BG_LD + lane]));
        }
        w1[lane] = cadd(cadd(a0, a1), cadd(a2, a3));
      }
      __syncwarp();
      if (lane < L) {
        const double2 cv = cmul(cconj(tau), v);
#pragma unroll 4
        for (int q = 1; q < BW; ++q) AB[(c0 + q) * LDB + (BW + lane - q)] = csub(Bs[lane * BG_LD + q], cmul(cv, w1[q]));
      }
    }
  } else if (wid == 2) {
    // two-sided update of the diagonal block: D <- H^H D H
    double2 y = make_double2(0, 0);
    if (lane < L) {
      double2 y1 = y, y2 = y, y3 = y;
      for (int q = 0; q < L; q += 4) {
        y = cadd(y, cmul(Ds[lane * BG_LD + q], vs[q]));
        if (q + 1 < L) y1 = cadd(y1, cmul(Ds[lane * BG_LD + q + 1], vs[q + 1]));
        if (q + 2 < L) y2 = cadd(y2, cmul(Ds[lane * BG_LD + q + 2], vs[q + 2]));
        if (q + 3 < L) y3 = cadd(y3, cmul(Ds[lane * BG_LD + q + 3], vs[q + 3]));
      }
      y = cadd(cadd(y, y1), cadd(y2, y3));
    }
    const double pv = warp_sum(cmulc(v, y).x);
    const double t2 = tau.x * tau.x + tau.y * tau.y;
    const double2 w = csub(cmul(tau, y), cscale(v, 0.5 * t2 * pv));
    w2[lane] = w;
    __syncwarp();
    if (lane < L)
#pragma unroll 4
      for (int q = 0; q <= lane; ++q) {
        double2 d = csub(Ds[lane * BG_LD + q], cadd(cmulc(w2[q], v), cmulc(vs[q], w)));
        if (q == lane) d.y = 0.0;
        AB[(r0 + q) * LDB + (lane - q)] = d;
      }
  } else if (L1 > 0 && lane < L1) {
    // right application to the block below: B1 <- B1 H
    double2 z = make_double2(0, 0), z1 = z, z2 = z, z3 = z;
    for (int q = 0; q < L; q += 4) {
      z = cadd(z, cmul(B1s[lane * BG_LD + q], vs[q]));
      if (q + 1 < L) z1 = cadd(z1, cmul(B1s[lane * BG_LD + q + 1], vs[q + 1]));
      if (q + 2 < L) z2 = cadd(z2, cmul(B1s[lane * BG_LD + q + 2], vs[q + 2]));
      if (q + 3 < L) z3 = cadd(z3, cmul(B1s[lane * BG_LD + q + 3], vs[q + 3]));
    }
    z = cadd(cadd(z, z1), cadd(z2, z3));
    const double2 tz = cmul(tau, z);
    // also in place: the next step's bulge block
#pragma unroll 4
    for (int q = 0; q < L; ++q) {
      const double2 nb = csub(B1s[lane * BG_LD + q], cmul(tz, cconj(vs[q])));
      AB[(r0 + q) * LDB + (L + lane - q)] = nb;
      B1s[lane * BG_LD + q] = nb;
    }
  }
}

__global__ void __launch_bounds__(B4_THREADS) k_bulge4(BulgeArgs a) {
  extern __shared__ __align__(16) double2 b4sm[];
  __shared__ int s_bad;
  const int tid = threadIdx.x;
  const long long W = (long long)gridDim.x;
  const long long N = a.N;
  const long long np = a.nprob;
  // same sweep order and wait rule as k_bulge, one CTA per sweep
  for (long long u = blockIdx.x; u < np * (N - 1); u += W) {
    const long long q = u % np, s = u / np;
    BulgeArgs b = a;
    b.AB = a.AB + q * a.ab_stride;
    unsigned int* prog = a.prog + q * a.prog_stride;
    const long long ns = nsteps_of(N, s);
    const long long nprev = (s > 0) ? nsteps_of(N, s - 1) : 0;
    double2* Bb = b4sm;                // roles of the three tiles rotate between steps
    double2* Db = b4sm + BW * BG_LD;
    double2* B1b = Db + BW * BG_LD;
    double2* tail = b4sm + 3 * BW * BG_LD;
    double2 gv[NGMAX];
    bool pre = false;
    for (long long t = 0; t < ns; ++t) {
      if (tid == 0) s_bad = (s > 0 && !wait_at_least(prog + s - 1, (unsigned int)min(t + 3, nprev), a.err)) ? 1 : 0;
      __syncthreads();
      if (s_bad) return;
      bulge_step4(b, s, t, Bb, Db, B1b, tail, gv, pre);
      // publish: the CTA barrier orders every thread's writes before the release store, issued
      // by warp 3 so that its latency overlaps thread 0's wait for the next step
      __syncthreads();
      if (tid == 96) st_release(prog + s, (unsigned int)(t + 1));
      pre = false;
      if (t + 1 < ns) {
        // Prefetch for step t + 1 (rows r0n = r0 + 32 on): its bulge block is this step's block
        // below (updated in place); its diagonal block, its block below and the velocity rows
        // are final already: the predecessor sweep's steps <= t + 2 that write them are done
        // (this step waited for t + 3), this step wrote none of them, and of the predecessor's
        // step t + 3 only the corner (31, 31) of the block below overlaps (read after the wait).
        // The successor sweep runs at most step t - 1 from now on and touches rows above.
        double2* tmp = Bb;
        Bb = B1b;
        B1b = tmp;
        const long long r0n = s + 1 + (t + 1) * BW;
        const int Ln = (int)min((long long)BW, N - r0n);
        const long long r1n = r0n + Ln;
        const int L1n = (r1n < N) ? (int)min((long long)BW, N - r1n) : 0;
        if (tid < 96) {
          for (int e = tid; e < BW * BW; e += 96) {
            const int i = e & 31, q = e >> 5;
            if (q < Ln) {
              const bool ok = i >= q && i < Ln;
              cpa16(Db + i * BG_LD + q, ok ? b.AB + (r0n + q) * LDB + (i - q) : b.AB, ok);
              if (!(i == BW - 1 && q == BW - 1 && Ln == BW && L1n == BW))
                cpa16(B1b + i * BG_LD + q, b.AB + (r0n + q) * LDB + (Ln + i - q), i < L1n);
            }
          }
          asm volatile("cp.async.commit_group;" ::: "memory");
        }
        if (tid < 32) {
#pragma unroll
          for (int al2 = 0; al2 < NGMAX; ++al2)
            gv[al2] = (al2 < a.ng && tid < Ln) ? __ldcg(a.g + (long long)al2 * N + r0n + tid) : make_double2(0, 0);
        }
        pre = true;
      }
    }
  }
}

__global__ void k_band_to_tridiag(const double2* __restrict__ AB, long long N, double* __restrict__ d,
                                  double* __restrict__ e) {
  const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (j >= N) return;
  d[j] = AB[j * LDB].x;
  if (j < N - 1) e[j] = AB[j * LDB + 1].x;
}

// ----------------------------------------------------------------------------- back-transform
// Stage-2 reflectors in reverse: sweeps from the last, each step after the next sweep has
// finished its steps up to t (the ranges are then disjoint); X (n x nvec, column-major).
__global__ void __launch_bounds__(32 * BG_WARPS, 1) k_bulge_back(const double2* __restrict__ A, long long N,
                                                                  const double2* __restrict__ tau2, double2* X, int nvec,
                                                                  unsigned int* prog, int* err) {
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long W = (long long)gridDim.x * BG_WARPS;
  for (long long u = (long long)blockIdx.x * BG_WARPS + wid; u < N - 1; u += W) {
    const long long s = N - 2 - u;
    const long long ns = nsteps_of(N, s);
    const long long nnext = (s + 1 < N - 1) ? nsteps_of(N, s + 1) : 0;
    for (long long t = 0; t < ns; ++t) {
      if (s + 1 < N - 1) {
        const unsigned int need = (unsigned int)min(t + 1, nnext);
        int bad = 0;
        if (lane == 0) bad = wait_at_least(prog + s + 1, need, err) ? 0 : 1;
        bad = __shfl_sync(0xffffffffu, bad, 0);
        if (bad) return;
      }
      const long long r0 = s + 1 + t * BW;
      const int L = (int)min((long long)BW, N - r0);
      const double2 v = (lane < L) ? A[(r0 + lane - s - 1) + (N - 1 - s) * N] : make_double2(0, 0);
      const double2 tau = tau2[tau2_offset(N, s) + t];
      for (int c = 0; c < nvec; ++c) {
        double2* xp = X + (long long)c * N + r0;
        const double2 xv = (lane < L) ? __ldcg(xp + lane) : make_double2(0, 0);
        const double2 sv = warp_sum2(cmulc(v, xv));   // v^H x
        if (lane < L) xp[lane] = csub(xv, cmul(tau, cmul(v, sv)));
      }
      __syncwarp();
      if (lane == 0) st_release(prog + s, (unsigned int)(t + 1));
    }
  }
}

// Stage-1 block reflectors in reverse: X[k0:] -= V (T (V^H X[k0:])).  V from the panel's
// columns of A (unit at row k0+q, v below, zero above).
constexpr int BT1_RB = 128;
__device__ __forceinline__ double2 panel_v(const double2* A, long long N, int j0, int k0, int q, long long r) {
  const long long rq = (long long)k0 + q;
  if (r < rq) return make_double2(0, 0);
  if (r == rq) return make_double2(1.0, 0.0);
  return A[r + (long long)(j0 + q) * N];
}
__global__ void __launch_bounds__(256) k_bt1_partial(const double2* __restrict__ A, long long N, int j0, int k0, int nref,
                                                     const double2* __restrict__ X, int nvec, double2* __restrict__ part) {
  // part[b][q + 32 c] = sum over this block's rows of conj(V[r][q]) X[r][c]
  const long long rb = (long long)k0 + (long long)blockIdx.x * BT1_RB;
  for (int e = threadIdx.x; e < 32 * nvec; e += 256) {
    const int q = e & 31, c = e >> 5;
    double2 t = make_double2(0, 0);
    if (q < nref)
      for (int i = 0; i < BT1_RB; ++i) {
        const long long r = rb + i;
        if (r >= N) break;
        t = cadd(t, cmulc(panel_v(A, N, j0, k0, q, r), X[r + (long long)c * N]));
      }
    part[(size_t)blockIdx.x * 32 * 32 + e] = t;
  }
}
__global__ void __launch_bounds__(1024) k_bt1_tmat(const double2* __restrict__ part, int nb, int nvec,
                                                   const double2* __restrict__ T, double2* __restrict__ Y) {
  __shared__ double2 sY[32 * 32];
  const int e = threadIdx.x;
  const int q = e & 31, c = e >> 5;
  double2 t = make_double2(0, 0);
  if (c < nvec)
    for (int b = 0; b < nb; ++b) t = cadd(t, part[(size_t)b * 32 * 32 + e]);
  sY[e] = t;
  __syncthreads();
  if (c < nvec) {   // (T Y)[q][c] = sum_{l >= q} T[q][l] Y[l][c]
    double2 s = make_double2(0, 0);
    for (int l = q; l < 32; ++l) s = cadd(s, cmul(T[q + 32 * l], sY[l + 32 * c]));
    Y[e] = s;
  }
}
__global__ void __launch_bounds__(256) k_bt1_apply(const double2* __restrict__ A, long long N, int j0, int k0, int nref,
                                                   double2* X, int nvec, const double2* __restrict__ Y) {
  __shared__ double2 sY[32 * 32];
  for (int e = threadIdx.x; e < 32 * nvec; e += 256) sY[e] = Y[e];
  __syncthreads();
  const long long r = (long long)k0 + (long long)blockIdx.x * 256 + threadIdx.x;
  if (r >= N) return;
  double2 vq[32];
#pragma unroll
  for (int q = 0; q < 32; ++q) vq[q] = (q < nref) ? panel_v(A, N, j0, k0, q, r) : make_double2(0, 0);
  for (int c = 0; c < nvec; ++c) {
    double2 t = make_double2(0, 0);
#pragma unroll
    for (int q = 0; q < 32; ++q) t = cadd(t, cmul(vq[q], sY[q + 32 * c]));
    X[r + (long long)c * N] = csub(X[r + (long long)c * N], t);
  }
}

}  // namespace

// Largest N whose panels fit the aggregate shared memory of the panel QR (one CTA per SM,
// at most PQ_MAX_R rows of the 32-wide panel each).
constexpr int PQ_MAX_R = 384;
constexpr long long LA_FOUR_FROM = 20000;   // N from which groups of four are used
constexpr int LOOKAHEAD = 4;   // largest number of panels applied per rank-2k update (K = 128)
// the look-ahead corrections stage K = 32 (group - 1) rows in shared memory (200 KB at 4)
static_assert(LOOKAHEAD >= 1 && LOOKAHEAD <= 4, "look-ahead groups of 1 to 4 panels");
// Group size per reduction: the wider update pays off where the trailing matrices are large
// (config 2, N = 36864: fours 11.75 s, pairs 11.86 s per step); at N = 8100 the update rate does
// not rise and the corrections cost more (fours 228 ms, pairs 223 ms per config-4 Q).
inline int lookahead_group(long long N) { return N >= LA_FOUR_FROM ? 4 : 2; }
static bool two_stage_fits(wtbg_ctx* ctx, long long N) {
  if (ctx->nsm <= 0) cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, ctx->device);
  return N > BW + 1 && (N + ctx->nsm - 1) / ctx->nsm <= PQ_MAX_R;
}

// The reduction used for the current matrix: two-stage for large N (auto) where it fits.
bool use_two_stage(wtbg_ctx* ctx) {
  const long long N = ctx->N;
  if (ctx->tri_mode == 1) return false;
  if (!two_stage_fits(ctx, N)) return false;
  if (ctx->tri_mode == 2) return true;
  return N >= 2048;
}

// Work buffers of the two-stage reduction for N (nband bands side by side for Q groups).
static int two_stage_buffers(wtbg_ctx* ctx, int nband) {
  const long long N = ctx->N;
  const int nsm = ctx->nsm > 0 ? ctx->nsm : 148;
  const long long npan = (N - BW - 1 + BW - 1) / BW;
  const long long nI = (N + 63) / 64;
  ENSURE(ctx->d, (size_t)N * 8);
  ENSURE(ctx->e, (size_t)N * 8);
  ENSURE(ctx->g, (size_t)N * 16 * NGMAX);
  ENSURE(ctx->Wp, (size_t)N * 16 * LOOKAHEAD * BW);
  ENSURE(ctx->t2V, (size_t)N * 16 * LOOKAHEAD * BW);
  ENSURE(ctx->t2X, (size_t)8 * BW * N * 16);
  ENSURE(ctx->t2D, (size_t)nI * 64 * 64 * 16);
  ENSURE(ctx->t2G, (size_t)nI * 1024 * 16 + 1024 * 16 + (size_t)nI * 2 * (LOOKAHEAD - 1) * 1024 * 16 +
                        (size_t)2 * (LOOKAHEAD - 1) * 1024 * 16);
  ENSURE(ctx->t2T, (size_t)std::max<long long>(npan, 1) * 1024 * 16);
  ENSURE(ctx->t2P, (size_t)nsm * (16 + 2 * 16 * BW + 16 * BW * BW + 16 * BW * NGMAX) + 4096 +
                        (size_t)std::max<long long>(npan, 1) * 4);
  ENSURE(ctx->t2AB, (size_t)nband * N * LDB * 16);
  ENSURE(ctx->t2prog, (size_t)nband * N * 4 + 64);
  ENSURE(ctx->triErr, 16);
  return 0;
}

// Stage 1 (dense -> band) of the context's matrix; the band goes to slot `band` of ctx->t2AB.
// ng velocity vectors in ctx->g follow the reflectors.
static int run_stage1(wtbg_ctx* ctx, int ng, int band) {
  const long long N = ctx->N;
  cudaStream_t s = ctx->stream;
  const int nsm = ctx->nsm > 0 ? ctx->nsm : 148;
  const long long npan = (N - BW - 1 + BW - 1) / BW;
  const long long nI = (N + 63) / 64;
  const int SMAX = 8;
  double2* A = ctx->H.as<double2>();
  double2* g = ctx->g.as<double2>();
  double2* Vp = ctx->t2V.as<double2>();
  double2* Wp = ctx->Wp.as<double2>();
  double2* Xpart = ctx->t2X.as<double2>();
  double2* Dsym = ctx->t2D.as<double2>();
  double2* Gpart = ctx->t2G.as<double2>();
  double2* Mbuf = Gpart + (size_t)nI * 1024;
  double2* Cpart = Mbuf + 1024;                                        // look-ahead correction partials
  double2* Cbuf = Cpart + (size_t)nI * 2 * (LOOKAHEAD - 1) * 1024;     // C1 (K x 32) then C2
  double2* Tbuf = ctx->t2T.as<double2>();
  char* pb = ctx->t2P.as<char>();
  double* partN = reinterpret_cast<double*>(pb);
  double2* partW = reinterpret_cast<double2*>(pb + (size_t)nsm * 16);   // 16-byte aligned for any SM count
  double2* partG = partW + (size_t)2 * nsm * BW;
  double2* partVg = partG + (size_t)nsm * BW * BW;
  double2* alpha = partVg + (size_t)nsm * BW * NGMAX;
  unsigned int* cnt = reinterpret_cast<unsigned int*>(alpha + 2 * BW);   // one barrier counter per panel launch
  int* err = ctx->triErr.as<int>();
  CK(cudaMemsetAsync(cnt, 0, (size_t)std::max<long long>(npan, 1) * 4, s));
  CK(cudaFuncSetAttribute(k_hemm2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HM_SMEM));
  CK(cudaFuncSetAttribute(k_xreduce, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)XR_SMEM));
  CK(cudaFuncSetAttribute(k_symdiag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SD_SMEM));
  // profiling: event pairs around the panel QR, the Hermitian product and the rank-2k update
  // of every panel (read after the stage), and around the stage
  const bool prof = ctx->profiling != 0;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  if (prof) {
    for (auto& e : ev) CK(cudaEventCreate(&e));
    if (int r = ensure_events(ctx, 6 * (size_t)std::max<long long>(npan, 1))) return r;
    cudaEventRecord(ev[0], s);
  }
  auto mark = [&](long long pnl, int k) {
    if (prof) cudaEventRecord(ctx->evpool[6 * pnl + k], s);
  };
  // Panel QR of panel pnl into V (its 32 columns), then X = A22 V (split K) and W.  Inside a
  // look-ahead group (K > 0) A22 still lacks the updates of the group's K/32 earlier panels
  // (Vacc, Wacc) and the product is corrected by -Vacc C1 - Wacc C2.
  auto panel = [&](long long pnl, double2* V, double2* Wout, int K) -> int {
    const int j0 = (int)(pnl * BW), k0 = j0 + BW;
    const long long m = N - k0;
    const int nref = (int)std::min<long long>(BW, m);
    // panel QR: G CTAs of R rows (at most 64 CTAs while the rows fit: the panel is latency-bound,
    // and fewer CTAs make the grid barrier and the cross-CTA reductions cheaper)
    const int R = (int)std::min<long long>(PQ_MAX_R, std::max<long long>(64, (m + 63) / 64));
    const int G = (int)((m + R - 1) / R);
    PanelArgs pa;
    pa.A = A;
    pa.N = N;
    pa.j0 = j0;
    pa.k0 = k0;
    pa.jb = BW;
    pa.nref = nref;
    pa.R = R;
    pa.RS = R | 1;
    pa.Vp = V;
    pa.Tout = Tbuf + (size_t)pnl * 1024;
    pa.g = g;
    pa.ng = ng;
    pa.partN = partN;
    pa.partW = partW;
    pa.partG = partG;
    pa.partVg = partVg;
    pa.alpha = alpha;
    pa.cnt = cnt + pnl;
    pa.err = err;
    const size_t psm = (size_t)BW * (R | 1) * 16;
    CK(cudaFuncSetAttribute(k_panel_qr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psm));
    if (G > PQ_MAXG) return set_err(ctx, WTBG_ERR_UNSUPPORTED, "panel QR: more CTAs than the column reduction holds");
    mark(pnl, 0);
    {
      void* args[] = {&pa};
      CK(cudaLaunchCooperativeKernel((const void*)k_panel_qr, dim3(G), dim3(PQ_THREADS), args, psm, s));
    }
    mark(pnl, 1);
    const int nIm = (int)((m + 63) / 64);
    k_symdiag<<<nIm, 256, SD_SMEM, s>>>(A, N, k0, Dsym);
    int S = (int)std::min<long long>(SMAX, std::max<long long>(1, (4LL * nsm + nIm - 1) / nIm));
    S = std::min(S, nIm);
    const int chunkJ = (nIm + S - 1) / S;
    S = (nIm + chunkJ - 1) / chunkJ;
    mark(pnl, 2);
    k_hemm2<<<dim3(nIm, S), 256, HM_SMEM, s>>>(A, N, k0, Dsym, V, nIm, chunkJ, Xpart);
    mark(pnl, 3);
    if (K > 0) {
      const size_t cps = ((size_t)K * CP_LD + 32 * CP_LD) * 16, xcs = ((size_t)2 * K * 32 + 2 * (size_t)K * 33) * 16;
      CK(cudaFuncSetAttribute(k_cpart, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cps));
      CK(cudaFuncSetAttribute(k_xcorr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xcs));
      k_cpart<<<dim3(nIm, 2), 256, cps, s>>>(N, k0, K, Vp, Wp, V, Cpart);
      k_creduce<<<(2 * K * 32 + 255) / 256, 256, 0, s>>>(Cpart, nIm, K, Cbuf);
      k_xcorr<<<(int)((m + 31) / 32), 256, xcs, s>>>(Xpart, N, k0, K, Vp, Wp, Cbuf);
      WTBG_COUNT(ctx, 3);
    }
    k_xreduce<<<nIm, 256, XR_SMEM, s>>>(Xpart, S, N, k0, Tbuf + (size_t)pnl * 1024, V, Wout, Gpart);
    k_mform<<<1, 1024, 0, s>>>(Gpart, nIm, Tbuf + (size_t)pnl * 1024, Mbuf);
    k_wform<<<(int)((m + 31) / 32), 256, 0, s>>>(N, k0, V, Mbuf, Wout);
    WTBG_COUNT(ctx, 6);
    CKL("two-stage panel");
    return 0;
  };
  // Panels in look-ahead groups of la (up to LOOKAHEAD): panel j of a group first gets the pending
  // updates of the group's earlier panels on its own 32 columns (strip), is factored, and forms
  // its product from the matrix that still lacks those updates (corrected); one rank-2k update
  // with K = 32 x (panels in the group) then applies the whole group to the trailing matrix.
  std::vector<double> her2k_flops(npan, 0.0);
  const int la = std::min(LOOKAHEAD, lookahead_group(N));
  for (long long p0 = 0; p0 < npan; p0 += la) {
    const int gsz = (int)std::min<long long>(la, npan - p0);
    for (int j = 0; j < gsz; ++j) {
      const long long pnl = p0 + j;
      if (j > 0) {
        const long long c0 = pnl * BW;   // the panel's first column (= the previous panel's k0)
        const long long mc = N - c0;
        const size_t sss = ((size_t)2 * 32 * j * 32 + (size_t)2 * 32 * j * 33) * 16;
        CK(cudaFuncSetAttribute(k_strip_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sss));
        mark(pnl - 1, 4);
        k_strip_update<<<(int)((mc + 31) / 32), 256, sss, s>>>(A, N, c0, 32 * j, Vp, Wp);
        WTBG_COUNT(ctx, 1);
        mark(pnl - 1, 5);
        her2k_flops[pnl - 1] = 8.0 * (double)mc * 32 * 2 * 32 * j;
      }
      if (int r = panel(pnl, Vp + (size_t)32 * j * N, Wp + (size_t)32 * j * N, 32 * j)) return r;
    }
    const long long pl = p0 + gsz - 1;
    const long long kl = (pl + 1) * BW;
    const long long ml = N - kl;
    const int Kg = 32 * (gsz - 1) + (int)std::min<long long>(BW, ml);
    mark(pl, 4);
    if (int r = launch_her2k_v(ctx, A, N, Wp, Vp, N, 0, Kg, kl)) return r;
    mark(pl, 5);
    her2k_flops[pl] = (double)ml * (ml + 1.0) * 0.5 * 16.0 * Kg;
  }
  k_band_extract<<<(unsigned)N, 128, 0, s>>>(A, N, ctx->t2AB.as<double2>() + (size_t)band * N * LDB);
  WTBG_COUNT(ctx, 1);
  CKL("k_band_extract");
  if (prof) {
    cudaEventRecord(ev[1], s);
    CK(cudaEventSynchronize(ev[1]));
    float t = 0.f;
    cudaEventElapsedTime(&t, ev[0], ev[1]);
    ctx->stats.stage1_ms += t;
    ctx->stats.tri_ms += t;
    for (long long pnl = 0; pnl < npan; ++pnl) {
      const double m = (double)(N - (pnl + 1) * BW), nref = std::min(m, (double)BW);
      float a = 0.f, b = 0.f, c = 0.f;
      cudaEventElapsedTime(&a, ctx->evpool[6 * pnl + 0], ctx->evpool[6 * pnl + 1]);
      cudaEventElapsedTime(&b, ctx->evpool[6 * pnl + 2], ctx->evpool[6 * pnl + 3]);
      cudaEventElapsedTime(&c, ctx->evpool[6 * pnl + 4], ctx->evpool[6 * pnl + 5]);
      ctx->stats.panel_ms += a;
      ctx->stats.hemm_ms += b;
      ctx->stats.hemm_flops += 8.0 * m * m * nref;
      ctx->stats.her2k_ms += c;   // rank-2k updates (K = 64 per pair) and the look-ahead strips
      ctx->stats.her2k_flops += her2k_flops[pnl];
      ctx->stats.her2k_launches += 1;
    }
    for (auto& e : ev) cudaEventDestroy(e);
  }
  return 0;
}

// Stage 2 (band -> tridiagonal) of nband bands of ctx->t2AB in one persistent launch; the
// tridiagonal forms go to dd/ee ([nband][N] each).  With store (one band only; ctx->tau must
// hold ceil_sum(N-1) entries) the ng velocity vectors follow the reflectors and the reflectors
// are kept for the eigenvector back-transform; without, only the band is reduced.
static int run_stage2(wtbg_ctx* ctx, int nband, int ng, bool store, double* dd, double* ee) {
  if (store && (nband != 1 || ctx->tau.bytes < (size_t)std::max<long long>(ceil_sum(ctx->N - 1), 1) * 16))
    return set_err(ctx, WTBG_ERR_STATE, "two-stage: reflector storage not sized");
  const long long N = ctx->N;
  cudaStream_t s = ctx->stream;
  const int nsm = ctx->nsm > 0 ? ctx->nsm : 148;
  double2* AB = ctx->t2AB.as<double2>();
  unsigned int* prog = ctx->t2prog.as<unsigned int>();
  const bool prof = ctx->profiling != 0;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  if (prof) {
    for (auto& e : ev) CK(cudaEventCreate(&e));
    cudaEventRecord(ev[0], s);
  }
  CK(cudaMemsetAsync(prog, 0, (size_t)nband * N * 4, s));
  BulgeArgs ba;
  ba.AB = AB;
  ba.N = N;
  ba.A = ctx->H.as<double2>();
  ba.tau2 = ctx->tau.as<double2>();
  ba.g = ctx->g.as<double2>();
  ba.ng = store ? ng : 0;
  ba.prog = prog;
  ba.err = ctx->triErr.as<int>();
  ba.store = store ? 1 : 0;
  ba.nprob = nband;
  ba.ab_stride = N * LDB;
  ba.prog_stride = N;
  const long long nsweep = (long long)nband * (N - 1);
  if (ctx->bulge_warp_mode) {   // one warp per sweep
    const size_t bsm = (size_t)BG_WARPS * BG_WARP_TILE * 16;
    CK(cudaFuncSetAttribute(k_bulge, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bsm));
    int per = 1;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_bulge, 32 * BG_WARPS, bsm));
    const int gb = (int)std::max<long long>(1, std::min<long long>((long long)nsm * std::max(per, 1),
                                                                    (nsweep + BG_WARPS - 1) / BG_WARPS));
    void* args[] = {&ba};
    CK(cudaLaunchCooperativeKernel((const void*)k_bulge, dim3(gb), dim3(32 * BG_WARPS), args, bsm, s));
  } else {   // one CTA of four warps per sweep
    CK(cudaFuncSetAttribute(k_bulge4, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)B4_SMEM));
    int per = 1;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_bulge4, B4_THREADS, B4_SMEM));
    const int gb = (int)std::max<long long>(1, std::min<long long>((long long)nsm * std::max(per, 1), nsweep));
    void* args[] = {&ba};
    CK(cudaLaunchCooperativeKernel((const void*)k_bulge4, dim3(gb), dim3(B4_THREADS), args, B4_SMEM, s));
  }
  for (int q = 0; q < nband; ++q)
    k_band_to_tridiag<<<(int)((N + 255) / 256), 256, 0, s>>>(AB + (size_t)q * N * LDB, N, dd + (size_t)q * N,
                                                              ee + (size_t)q * N);
  WTBG_COUNT(ctx, 1 + nband);
  CKL("two-stage bulge chasing");
  if (prof) {
    cudaEventRecord(ev[1], s);
    CK(cudaEventSynchronize(ev[1]));
    float t = 0.f;
    cudaEventElapsedTime(&t, ev[0], ev[1]);
    ctx->stats.stage2_ms += t;
    ctx->stats.tri_ms += t;
    for (auto& e : ev) cudaEventDestroy(e);
  }
  return 0;
}

int run_tridiagonalise2(wtbg_ctx* ctx) {
  const long long N = ctx->N;
  cudaStream_t s = ctx->stream;
  if (int r = two_stage_buffers(ctx, 1)) return r;
  ENSURE(ctx->tau, (size_t)std::max<long long>(ceil_sum(N - 1), 1) * 16);
  CK(cudaMemsetAsync(ctx->triErr.p, 0, 4, s));
  double2* g = ctx->g.as<double2>();
  // velocity vectors g (as the one-stage reduction)
  const int ng = ctx->have_velocity ? (ctx->temp_on ? 10 : 5) : 0;
  ctx->ng = ctx->have_velocity ? ng : 5;
  if (ctx->have_velocity && ctx->temp_on) {
    if (int r = fill_g_vectors(ctx, g)) return r;
  } else if (ctx->have_velocity) {
    CK(cudaMemcpyAsync(g, ctx->h.p, (size_t)N * 16 * 5, cudaMemcpyDeviceToDevice, s));
  } else {
    CK(cudaMemsetAsync(g, 0, (size_t)N * 16 * 5, s));
  }
  if (int r = run_stage1(ctx, ng, 0)) return r;
  if (int r = run_stage2(ctx, 1, ng, true, ctx->d.as<double>(), ctx->e.as<double>())) return r;
  ctx->tri_two = true;
  return 0;
}

// Q groups of the exciton band structure (eigenvalues only): group_begin sizes the work
// buffers for nq bands, group_add runs stage 1 of the matrix just built into band slot i, and
// group_finish chases all nq bands in one persistent launch; the tridiagonal forms of the group
// land in dd/ee ([nq][N] each).
int two_stage_group_begin(wtbg_ctx* ctx, int nq) {
  if (int r = two_stage_buffers(ctx, nq)) return r;
  ENSURE(ctx->t2de, (size_t)2 * nq * ctx->N * 8);
  CK(cudaMemsetAsync(ctx->triErr.p, 0, 4, ctx->stream));
  return 0;
}
int two_stage_group_add(wtbg_ctx* ctx, int slot) { return run_stage1(ctx, 0, slot); }
int two_stage_group_finish(wtbg_ctx* ctx, int nq, double** dd, double** ee) {
  *dd = ctx->t2de.as<double>();
  *ee = *dd + (size_t)nq * ctx->N;
  if (int r = run_stage2(ctx, nq, 0, false, *dd, *ee)) return r;
  ctx->tri_two = false;   // no reflectors kept: exciton vectors need a wtbg_bse_solve
  return 0;
}

// Exciton vectors through both stages: X <- Q1 (Q2 X), Q2 the bulge-chasing reflectors in
// reverse, Q1 the panels' block reflectors in reverse.
int run_backtransform2(wtbg_ctx* ctx, double2* X, int nvec) {
  const long long N = ctx->N;
  cudaStream_t s = ctx->stream;
  const int nsm = ctx->nsm > 0 ? ctx->nsm : 148;
  unsigned int* prog = ctx->t2prog.as<unsigned int>();
  int* err = ctx->triErr.as<int>();
  CK(cudaMemsetAsync(prog, 0, (size_t)N * 4, s));
  CK(cudaMemsetAsync(err, 0, 4, s));
  const long long nsweep = N - 1;
  const int gb = (int)std::max<long long>(1, std::min<long long>(nsm, (nsweep + BG_WARPS - 1) / BG_WARPS));
  {
    const double2* A = ctx->H.as<double2>();
    const double2* tau2 = ctx->tau.as<double2>();
    long long NN = N;
    void* args[] = {(void*)&A, (void*)&NN, (void*)&tau2, (void*)&X, (void*)&nvec, (void*)&prog, (void*)&err};
    CK(cudaLaunchCooperativeKernel((const void*)k_bulge_back, dim3(gb), dim3(32 * BG_WARPS), args, 0, s));
  }
  const long long npan = (N - BW - 1 + BW - 1) / BW;
  const int nbmax = (int)((N + BT1_RB - 1) / BT1_RB);
  ENSURE(ctx->t2G, (size_t)nbmax * 1024 * 16 + 1024 * 16);
  double2* part = ctx->t2G.as<double2>();
  double2* Y = part + (size_t)nbmax * 1024;
  for (long long pnl = npan - 1; pnl >= 0; --pnl) {
    const int j0 = (int)(pnl * BW), k0 = j0 + BW;
    const long long m = N - k0;
    const int nref = (int)std::min<long long>(BW, m);
    const int nb = (int)((m + BT1_RB - 1) / BT1_RB);
    k_bt1_partial<<<nb, 256, 0, s>>>(ctx->H.as<double2>(), N, j0, k0, nref, X, nvec, part);
    k_bt1_tmat<<<1, 1024, 0, s>>>(part, nb, nvec, ctx->t2T.as<double2>() + (size_t)pnl * 1024, Y);
    k_bt1_apply<<<(int)((m + 255) / 256), 256, 0, s>>>(ctx->H.as<double2>(), N, j0, k0, nref, X, nvec, Y);
  }
  WTBG_COUNT(ctx, 1 + 3 * npan);
  CKL("two-stage back-transform");
  int herr = 0;
  CK(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (herr) return set_err(ctx, WTBG_ERR_CUDA, "back-transform: a sweep wait timed out");
  return 0;
}
