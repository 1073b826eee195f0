// Kernel (c), stage 2: eigenvalues and oscillator strengths of the real symmetric
// tridiagonal T = Q^H H Q produced by tridiag.cu.
//
// Reference: ZHEEV('V','U') + dielbsev/dielbsep (subprograms/bse_solver-tool-diel.f90:485-602,
// subroutines/bse_subs.f90:278-378).  The oscillator strength of exciton n is
//   f_n = |sum_j A_jn h_j|^2 = |z_n^T g|^2,  g = Q^T h,  A = Q Z,
// so after the reduction only the tridiagonal eigenvectors z_n are needed, and only inside
// the dot products with the five g vectors.
//   * eigenvalues: one coarse round of Sturm counts at 32769 points of the Gershgorin interval
//     gives every eigenvalue index its starting cell; then Sturm-count multisection, L lanes
//     per eigenvalue index (L = 1: bisection), to full precision;
//   * eigenvectors: inverse iteration with a partial-pivoting tridiagonal LU, three steps
//     from a deterministic pseudo-random start vector; eigenvalues closer than
//     1e-7 * ||T|| form a cluster that one thread processes in sequence with modified
//     Gram-Schmidt against the earlier members (so degenerate excitons get orthogonal
//     vectors); the vectors live in a chunked workspace laid out [k][slot] so that the
//     threads' accesses coalesce;
//   * the dot products with g are fused into the last pass over each vector.
// Selected exciton eigenvectors (BSE_WF) are back-transformed A_n = Q z_n panel by panel
// with the compact-WY form I - V T V^H of each panel's reflectors.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "common.cuh"

namespace {

constexpr int NG = 10;   // largest number of reduced h vectors (5, or 10 with temperature)

__device__ __forceinline__ int sturm_count(const double* __restrict__ d, const double* __restrict__ e2, long long n,
                                           double x, double pivmin) {
  int cnt = 0;
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  cnt += (q < 0.0);
  for (long long i = 1; i < n; ++i) {
    q = (d[i] - x) - e2[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    cnt += (q < 0.0);
  }
  return cnt;
}

__global__ void k_e2(const double* e, long long n, double* e2) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n - 1) e2[i] = e[i] * e[i];
}

// Multisection: L consecutive lanes (L a power of two, L <= 32) share eigenvalue m and, per
// round, take Sturm counts at L interior points of its interval [a, b]; the new interval runs
// from the highest point with count <= m to the next point (or b), so count(a) <= m < count(b)
// holds whatever the counts at the other points.  A round divides the interval by L + 1 (by 2,
// at the midpoint, for L = 1: plain bisection), so the chain of dependent Sturm passes per
// eigenvalue is log2(L + 1) times shorter, for L times more total passes; the host picks L.
// Stopping rule as in bisection: width <= 2 eps max(|a|, |b|) + pivmin, or no double between.
// Coarse round: Sturm counts at the P + 1 points x_j = lo + (hi - lo) j / P of the Gershgorin
// interval (count 0 at lo and n at hi by construction), one thread per point.
constexpr int BIS_P = 32768;
__global__ void k_bisect_grid(const double* __restrict__ d, const double* __restrict__ e2, long long n, double lo,
                              double hi, double pivmin, double* __restrict__ xg, int* __restrict__ cg) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j > BIS_P) return;
  const double x = (j == BIS_P) ? hi : lo + (hi - lo) * ((double)j / (double)BIS_P);
  xg[j] = x;
  cg[j] = (j == 0) ? 0 : (j == BIS_P ? (int)n : sturm_count(d, e2, n, x, pivmin));
}

__global__ void __launch_bounds__(128) k_bisect(const double* __restrict__ d, const double* __restrict__ e2, long long n,
                                                const double* __restrict__ xg, const int* __restrict__ cg,
                                                double pivmin, int L, double* lam) {
  const long long gt = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long m = gt / L;
  const int lane = threadIdx.x & 31, sl = lane & (L - 1), base = lane - sl;
  const bool active = m < n;
  // start from the coarse cell [x_j, x_{j+1}] with count(x_j) <= m < count(x_{j+1}) (binary
  // search keeping that invariant; cg[0] = 0 <= m < n = cg[P])
  double a = xg[0], b = xg[BIS_P];
  if (active) {
    int jl = 0, jh = BIS_P;
    while (jh - jl > 1) {
      const int jm = (jl + jh) >> 1;
      if (cg[jm] <= m) jl = jm;
      else jh = jm;
    }
    a = xg[jl];
    b = xg[jh];
  }
  for (int it = 0; it < 256; ++it) {
    const double mid = 0.5 * (a + b);
    const bool done = !active || !(mid > a && mid < b) || (b - a <= 2.0 * DBL_EPSILON * fmax(fabs(a), fabs(b)) + pivmin);
    if (__all_sync(0xffffffffu, done)) break;
    const double x = (L == 1) ? mid : a + (b - a) * ((double)(sl + 1) / (double)(L + 1));
    const bool le = !done && sturm_count(d, e2, n, x, pivmin) <= m;
    const unsigned gb = (__ballot_sync(0xffffffffu, le) >> base) & (L == 32 ? 0xffffffffu : ((1u << L) - 1u));
    const int jhi = gb ? 31 - __clz(gb) : -1;   // highest point with count <= m
    const double xa = __shfl_sync(0xffffffffu, x, base + max(jhi, 0));
    const double xb = __shfl_sync(0xffffffffu, x, base + min(jhi + 1, L - 1));
    if (!done) {
      if (jhi >= 0) a = xa;
      if (jhi + 1 < L) b = xb;
    }
  }
  if (active && sl == 0) lam[m] = 0.5 * (a + b);
}

// Lanes per eigenvalue for k_bisect.  A round costs one Sturm pass (n dependent steps of about
// 170 cycles) when the SM sub-partitions are idle, and n L / 32 warp passes of about 50 issue
// cycles per step spread over 4 nsm sub-partitions when they are full; after the coarse round
// (15 bits) rounds ~ 38 / log2(L+1).  (Constants fitted to B200 timings at N = 2304 and 9216
// over L = 4 .. 32.)
int bisect_lanes(long long n, int nsm) {
  int best = 1;
  double bt = 1e300;
  for (int L = 1; L <= 32; L *= 2) {
    const double rounds = std::ceil(38.0 / std::log2((double)L + 1.0));
    const double lat = 170.0 * (double)n;
    const double thr = 50.0 * (double)n * (double)n * (double)L / 32.0 / (4.0 * std::max(nsm, 1));
    const double t = rounds * std::max(lat, thr);
    if (t < bt) {
      bt = t;
      best = L;
    }
  }
  return best;
}

__device__ __forceinline__ double start_value(long long m, long long k) {
  unsigned long long z = (unsigned long long)m * 0x9E3779B97F4A7C15ull + (unsigned long long)k * 0xD1B54A32D192ED03ull + 0x632BE59BD9B4E019ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return ((double)(z >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0;
}

struct InvArgs {
  const double* d;
  const double* e;
  long long n;
  const double* lam;
  const int* csize;     // cluster size at a leader index, 0 for non-leaders
  long long m0;         // first eigenvalue index of the chunk
  long long m1;         // one past the last eigenvalue index of the chunk
  int M;                // slots in the chunk
  double* ws;           // 4 * n * M
  double pert;          // eps * ||T||: pivot floor
  const double2* g;     // [ng][n]: h (x, y, z, sp, sm) [, h * f with temperature]
  int ng;
  double* act;          // [8][n]
  int dtfull, cpol;
  double* zsel;         // selected vectors (column-major n x nsel) or null
  long long zs0, zs1;
};

constexpr int SB = 8;   // inverse-iteration steps whose loads are issued together

__global__ void __launch_bounds__(64) k_inviter(InvArgs a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.M) return;
  const long long m = a.m0 + j;
  if (m >= a.m1 || m >= a.n) return;
  const int cs = a.csize[m];
  if (cs == 0) return;
  const long long n = a.n;
  const int M = a.M;
  // Four disjoint slices of the workspace, laid out [k][slot]: each step of the elimination and
  // of the substitution is one link of a chain through a division, while its workspace loads
  // (one DRAM round trip each) do not depend on the chain; so the loads of SB steps are issued
  // together before the SB dependent steps run (same arithmetic, one round trip per SB steps).
  double* __restrict__ X = a.ws;
  double* __restrict__ U1 = a.ws + n * M;
  double* __restrict__ U2 = a.ws + 2 * n * M;
  double* __restrict__ U3 = a.ws + 3 * n * M;
  const double* __restrict__ dd_ = a.d;
  const double* __restrict__ ee_ = a.e;
  const double pert = a.pert;
  for (int s = 0; s < cs; ++s) {
    const long long mm = m + s;
    const int jj = j + s;
    const double lam = a.lam[mm];
    double sc = 1.0;
    for (long long k = 0; k < n; ++k) X[k * M + jj] = start_value(mm, k);
    for (int it = 0; it < 3; ++it) {
      // factor T - lam I with partial pivoting, eliminating the right-hand side on the fly
      double diag = dd_[0] - lam;
      double sup = (n > 1) ? ee_[0] : 0.0;
      double cur = X[jj] * sc;
      for (long long k0 = 0; k0 < n - 1; k0 += SB) {
        // the block's operands first (independent of the chain), then its SB dependent steps
        double xs[SB], es[SB + 1], ds[SB];
#pragma unroll
        for (int q = 0; q < SB; ++q) {
          const long long k = k0 + q;
          if (k < n - 1) {
            xs[q] = X[(k + 1) * M + jj];
            es[q] = ee_[k];
            ds[q] = dd_[k + 1];
          }
        }
        es[SB] = (k0 + SB < n - 1) ? ee_[k0 + SB] : 0.0;
#pragma unroll
        for (int q = 0; q < SB; ++q) {
          const long long k = k0 + q;
          if (k >= n - 1) break;
          const double sub = es[q];
          const double nd = ds[q] - lam;
          const double nsup = (k + 1 < n - 1) ? es[q + 1] : 0.0;
          const double nxt = xs[q] * sc;
          if (fabs(diag) >= fabs(sub)) {
            if (fabs(diag) < pert) diag = copysign(pert, diag);
            const double mult = sub / diag;
            U1[k * M + jj] = diag;
            U2[k * M + jj] = sup;
            U3[k * M + jj] = 0.0;
            X[k * M + jj] = cur;
            cur = nxt - mult * cur;
            diag = nd - mult * sup;
            sup = nsup;
          } else {
            const double mult = diag / sub;
            U1[k * M + jj] = sub;
            U2[k * M + jj] = nd;
            U3[k * M + jj] = nsup;
            X[k * M + jj] = nxt;
            cur = cur - mult * nxt;
            diag = sup - mult * nd;
            sup = -mult * nsup;
          }
        }
      }
      if (fabs(diag) < pert) diag = copysign(pert, diag);
      // back substitution (U1 of the last row kept in a register)
      double x2 = 0.0, x1 = cur / diag;
      X[(n - 1) * M + jj] = x1;
      double nrm = x1 * x1;
      for (long long kb = n - 2; kb >= 0; kb -= SB) {
        double xs[SB], u1[SB], u2[SB], u3[SB];
#pragma unroll
        for (int q = 0; q < SB; ++q) {
          const long long k = kb - q;
          if (k >= 0) {
            xs[q] = X[k * M + jj];
            u1[q] = U1[k * M + jj];
            u2[q] = U2[k * M + jj];
            u3[q] = U3[k * M + jj];
          }
        }
#pragma unroll
        for (int q = 0; q < SB; ++q) {
          const long long k = kb - q;
          if (k < 0) break;
          const double xk = (xs[q] - u2[q] * x1 - u3[q] * x2) / u1[q];
          X[k * M + jj] = xk;
          nrm += xk * xk;
          x2 = x1;
          x1 = xk;
        }
      }
      sc = 1.0 / sqrt(nrm);
      // orthogonalise against the earlier members of the cluster (normalised, in slots j..jj-1)
      if (s > 0) {
        for (int t = 0; t < s; ++t) {
          double dot = 0.0;
          for (long long k = 0; k < n; ++k) dot += X[k * M + jj] * X[k * M + j + t];
          for (long long k = 0; k < n; ++k) X[k * M + jj] -= dot * X[k * M + j + t];
        }
        double n2 = 0.0;
        for (long long k = 0; k < n; ++k) n2 += X[k * M + jj] * X[k * M + jj];
        sc = 1.0 / sqrt(n2);
      }
    }
    // final pass: normalise and accumulate the oscillator dot products
    double2 sg[NG];
#pragma unroll
    for (int al = 0; al < NG; ++al) sg[al] = make_double2(0, 0);
    const bool keep = (a.zsel != nullptr && mm >= a.zs0 && mm <= a.zs1);
    const int ng = a.ng;
    for (long long k0 = 0; k0 < n; k0 += SB) {
      double xs[SB];
#pragma unroll
      for (int q = 0; q < SB; ++q)
        if (k0 + q < n) xs[q] = X[(k0 + q) * M + jj];
#pragma unroll
      for (int q = 0; q < SB; ++q) {
        const long long k = k0 + q;
        if (k >= n) break;
        const double x = xs[q] * sc;
        X[k * M + jj] = x;
#pragma unroll
        for (int al = 0; al < NG; ++al) {
          if (al < ng) {
            const double2 gk = a.g[al * n + k];
            sg[al].x += x * gk.x;
            sg[al].y += x * gk.y;
          }
        }
        if (keep) a.zsel[(mm - a.zs0) * n + k] = x;
      }
    }
    // act(a, b) = Re[(z^T g_a) conj(z^T g'_b)], g' = g (dielbsev/dielbsep) or the f-weighted
    // vectors with temperature (dielbseptemp)
    const int o = (ng == 10) ? 5 : 0;
    auto re = [&](int p, int q) { return sg[p].x * sg[o + q].x + sg[p].y * sg[o + q].y; };
    double* act = a.act;
    act[0 * n + mm] = re(0, 0);
    act[1 * n + mm] = re(1, 1);
    act[2 * n + mm] = re(2, 2);
    act[3 * n + mm] = a.dtfull ? re(0, 1) : 0.0;
    act[4 * n + mm] = a.dtfull ? re(0, 2) : 0.0;
    act[5 * n + mm] = a.dtfull ? re(1, 2) : 0.0;
    act[6 * n + mm] = a.cpol ? re(3, 3) : 0.0;
    act[7 * n + mm] = a.cpol ? re(4, 4) : 0.0;
  }
}

// ---- back-transform of selected vectors: X <- Q X, Q = H_0 H_1 ... H_{n-2}
constexpr int PB = WTBG_PANEL;
constexpr int BT_RB = 256;

// partials of G = V^H V (PB x PB) and P = V^H X (PB x nv) over row blocks
__global__ void __launch_bounds__(BT_RB) k_bt_gram(const double2* A, long long n, int j0, int jb, const double2* X, int nvec,
                                                  double2* part) {
  extern __shared__ double2 sh[];
  const int tid = threadIdx.x;
  const int ncols = jb + nvec;
  const long long r = (long long)j0 + 1 + (long long)blockIdx.x * BT_RB + tid;
  // load this row of V (jb) and X (nvec)
  double2 vrow[PB];
#pragma unroll
  for (int q = 0; q < PB; ++q) {
    double2 v = make_double2(0, 0);
    if (q < jb && r < n && r >= (long long)j0 + q + 1) v = A[r + (long long)(j0 + q) * n];
    vrow[q] = v;
  }
  // each thread accumulates its row's outer products into shared memory via a block reduction
  double2* acc = sh;  // [jb][ncols]
  for (int it = tid; it < jb * ncols; it += BT_RB) acc[it] = make_double2(0, 0);
  __syncthreads();
  for (int qi = 0; qi < jb; ++qi) {
    for (int cj = 0; cj < ncols; ++cj) {
      double2 rhs = make_double2(0, 0);
      if (r < n) {
        if (cj < jb) rhs = vrow[cj];
        else rhs = X[(long long)(cj - jb) * n + r];
      }
      double2 t = cmulc(vrow[qi], rhs);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        t.x += __shfl_xor_sync(0xffffffffu, t.x, o);
        t.y += __shfl_xor_sync(0xffffffffu, t.y, o);
      }
      if ((tid & 31) == 0) {
        atomicAdd(&acc[qi * ncols + cj].x, t.x);
        atomicAdd(&acc[qi * ncols + cj].y, t.y);
      }
    }
  }
  __syncthreads();
  for (int it = tid; it < jb * ncols; it += BT_RB) part[(long long)blockIdx.x * PB * (PB + 64) + it] = acc[it];
}

// reduce partials, build T (zlarft forward/columnwise), Y = T P
__global__ void k_bt_tmat(const double2* part, int nparts, int jb, int nvec, const double2* tau, int j0, double2* Y) {
  __shared__ double2 G[PB][PB], Tm[PB][PB], P[PB][32];
  const int tid = threadIdx.x;
  const int ncols = jb + nvec;
  for (int it = tid; it < jb * ncols; it += blockDim.x) {
    double2 s = make_double2(0, 0);
    for (int k = 0; k < nparts; ++k) s = cadd(s, part[(long long)k * PB * (PB + 64) + it]);
    const int qi = it / ncols, cj = it % ncols;
    if (cj < jb) G[qi][cj] = s;
    else P[qi][cj - jb] = s;
  }
  __syncthreads();
  if (tid == 0) {
    for (int i = 0; i < jb; ++i) {
      const double2 ti = tau[j0 + i];
      Tm[i][i] = ti;
      // T(0:i, i) = -tau_i * T(0:i,0:i) * G(0:i, i)
      double2 tmp[PB];
      for (int r = 0; r < i; ++r) tmp[r] = cscale(cmul(ti, G[r][i]), -1.0);
      for (int r = 0; r < i; ++r) {
        double2 s = make_double2(0, 0);
        for (int c = r; c < i; ++c) s = cadd(s, cmul(Tm[r][c], tmp[c]));
        Tm[r][i] = s;
      }
      for (int r = i + 1; r < jb; ++r) Tm[r][i] = make_double2(0, 0);
    }
  }
  __syncthreads();
  for (int it = tid; it < jb * nvec; it += blockDim.x) {
    const int r = it / nvec, c = it % nvec;
    double2 s = make_double2(0, 0);
    for (int k = r; k < jb; ++k) s = cadd(s, cmul(Tm[r][k], P[k][c]));
    Y[r * 64 + c] = s;
  }
}

__global__ void k_bt_apply(const double2* A, long long n, int j0, int jb, double2* X, int nvec, const double2* Y) {
  const long long r = (long long)j0 + 1 + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= n) return;
  for (int c = 0; c < nvec; ++c) {
    double2 s = make_double2(0, 0);
    for (int q = 0; q < jb; ++q) {
      if (r < (long long)j0 + q + 1) continue;
      s = cadd(s, cmul(A[r + (long long)(j0 + q) * n], Y[q * 64 + c]));
    }
    X[(long long)c * n + r] = csub(X[(long long)c * n + r], s);
  }
}

__global__ void k_real_to_complex(const double* z, double2* X, long long cnt) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < cnt) X[i] = make_double2(z[i], 0.0);
}

// rotate each vector so that its last component is real and >= 0 (ZHEEV 'U' convention)
// each vector times conj(last)/|last|: the last component becomes real >= 0 (exactly real, as
// ZHEEV('V','U') returns it).  The last component is read before any thread writes.
__global__ void k_gauge_last(double2* X, long long n, int nvec) {
  const int c = blockIdx.x;
  if (c >= nvec) return;
  __shared__ double2 s_last;
  if (threadIdx.x == 0) s_last = X[(long long)c * n + n - 1];
  __syncthreads();
  const double2 last = s_last;
  const double r = hypot(last.x, last.y);
  double2 ph = make_double2(1, 0);
  if (r > 0) ph = make_double2(last.x / r, -last.y / r);
  for (long long k = threadIdx.x; k < n; k += blockDim.x) {
    double2 v = cmul(X[(long long)c * n + k], ph);
    if (k == n - 1) v = make_double2(r, 0.0);
    X[(long long)c * n + k] = v;
  }
}

}  // namespace

static int tridiagonal_solve_body(wtbg_ctx* ctx, int dtfull, int cpol, bool vectors);

// Eigenvalues (bisection) and, with vectors, the fused oscillator sums of the tridiagonal
// form; timed as a whole when profiling.
int run_tridiagonal_solve(wtbg_ctx* ctx, int dtfull, int cpol, bool vectors) {
  if (!ctx->profiling) return tridiagonal_solve_body(ctx, dtfull, cpol, vectors);
  if (int r = ensure_events(ctx, 2)) return r;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  cudaEventRecord(e0, ctx->stream);
  const int r = tridiagonal_solve_body(ctx, dtfull, cpol, vectors);
  cudaEventRecord(e1, ctx->stream);
  cudaEventSynchronize(e1);
  float t = 0.f;
  if (!r && cudaEventElapsedTime(&t, e0, e1) == cudaSuccess) ctx->stats.tdsolve_ms += t;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return r;
}

static int tridiagonal_solve_body(wtbg_ctx* ctx, int dtfull, int cpol, bool vectors) {
  const long long n = ctx->N;
  cudaStream_t s = ctx->stream;
  std::vector<double> hd(n), he(n > 1 ? n - 1 : 1, 0.0);
  CK(cudaMemcpyAsync(hd.data(), ctx->d.as<double>(), n * 8, cudaMemcpyDeviceToHost, s));
  if (n > 1) CK(cudaMemcpyAsync(he.data(), ctx->e.as<double>(), (n - 1) * 8, cudaMemcpyDeviceToHost, s));
  int tri_err = 0;
  if (ctx->triErr.p) CK(cudaMemcpyAsync(&tri_err, ctx->triErr.p, 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (tri_err) return set_err(ctx, WTBG_ERR_CUDA, "tridiagonalise: a mat-vec pipeline wait timed out");
  double lo = hd[0], hi = hd[0], emax2 = 0.0;
  for (long long i = 0; i < n; ++i) {
    const double r = (i > 0 ? fabs(he[i - 1]) : 0.0) + (i < n - 1 ? fabs(he[i]) : 0.0);
    lo = std::min(lo, hd[i] - r);
    hi = std::max(hi, hd[i] + r);
    if (i < n - 1) emax2 = std::max(emax2, he[i] * he[i]);
  }
  const double tnorm = std::max(fabs(lo), fabs(hi));
  const double pivmin = DBL_MIN * std::max(1.0, emax2);
  // widen the Gershgorin interval slightly so that the extreme eigenvalues are interior
  const double pad = 2.0 * DBL_EPSILON * tnorm + 4.0 * pivmin + 1e-300;
  lo -= pad;
  hi += pad;
  ENSURE(ctx->lam, (size_t)n * 8);
  ENSURE(ctx->tmp2, (size_t)n * 8 + 64);
  double* e2 = ctx->tmp2.as<double>();
  if (n > 1) {
    k_e2<<<(int)((n + 255) / 256), 256, 0, s>>>(ctx->e.as<double>(), n, e2); WTBG_COUNT(ctx, 1);
    CKL("k_e2");
  }
  if (ctx->nsm <= 0) cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, ctx->device);
  const int lanes = bisect_lanes(n, ctx->nsm);
  ENSURE(ctx->bgrid, (size_t)(BIS_P + 1) * (8 + 4) + 64);
  double* xg = ctx->bgrid.as<double>();
  int* cg = reinterpret_cast<int*>(xg + BIS_P + 1);
  k_bisect_grid<<<(BIS_P + 1 + 255) / 256, 256, 0, s>>>(ctx->d.as<double>(), e2, n, lo, hi, pivmin, xg, cg);
  CKL("k_bisect_grid");
  k_bisect<<<(int)((n * lanes + 127) / 128), 128, 0, s>>>(ctx->d.as<double>(), e2, n, xg, cg, pivmin, lanes,
                                                       ctx->lam.as<double>()); WTBG_COUNT(ctx, 2);
  CKL("k_bisect");
  ctx->lam_host.resize(n);
  CK(cudaMemcpyAsync(ctx->lam_host.data(), ctx->lam.as<double>(), n * 8, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (!vectors) return 0;

  // clusters (host): leaders carry the cluster size
  const std::vector<double>& L = ctx->lam_host;
  const double ctol = 1e-7 * std::max(1.0, tnorm);
  std::vector<int> csize(n, 0);
  long long maxc = 1;
  for (long long i = 0; i < n;) {
    long long jx = i + 1;
    while (jx < n && L[jx] - L[jx - 1] <= ctol) ++jx;
    csize[i] = (int)(jx - i);
    maxc = std::max(maxc, jx - i);
    i = jx;
  }
  // chunk size: the vectors of one launch run their chains side by side, so one launch for all
  // of them where the workspace fits (43.5 GB at N = 36864), else chunks
  size_t freeb = 0, totb = 0;
  CK(cudaMemGetInfo(&freeb, &totb));
  const double budget = std::min((double)freeb * 0.6 + (double)ctx->ws.bytes, 96e9);
  long long M = (long long)(budget / (4.0 * 8.0 * (double)n));
  M = std::max<long long>(M, maxc);
  M = std::min<long long>(M, n);
  M = std::max<long long>(M, 1);
  ENSURE(ctx->ws, (size_t)4 * 8 * n * M);
  ENSURE(ctx->act, (size_t)8 * 8 * n);
  ENSURE(ctx->csz, (size_t)n * 4 + 64);
  CK(cudaMemcpyAsync(ctx->csz.as<int>(), csize.data(), n * 4, cudaMemcpyHostToDevice, s));
  ctx->csize_host = csize;
  ctx->tnorm = tnorm;
  InvArgs a;
  a.d = ctx->d.as<double>();
  a.e = ctx->e.as<double>();
  a.n = n;
  a.lam = ctx->lam.as<double>();
  a.csize = ctx->csz.as<int>();
  a.ws = ctx->ws.as<double>();
  a.pert = DBL_EPSILON * std::max(tnorm, DBL_MIN);
  a.g = ctx->g.as<double2>();
  a.ng = ctx->ng;
  a.act = ctx->act.as<double>();
  a.dtfull = dtfull;
  a.cpol = cpol;
  a.zsel = nullptr;
  a.zs0 = -1;
  a.zs1 = -1;
  for (long long m0 = 0; m0 < n;) {
    // end the chunk at a cluster start
    long long m1 = std::min(n, m0 + M);
    if (m1 < n) {
      while (m1 > m0 && csize[m1] == 0) --m1;
      if (m1 == m0) m1 = std::min(n, m0 + M);
    }
    a.m0 = m0;
    a.m1 = m1;
    a.M = (int)M;
    const int cnt = (int)(m1 - m0);
    k_inviter<<<(cnt + 63) / 64, 64, 0, s>>>(a); WTBG_COUNT(ctx, 1);
    CKL("k_inviter");
    m0 = m1;
  }
  return 0;
}

int run_eigvecs(wtbg_ctx* ctx, int n0, int n1, double2* d_out) {
  const long long n = ctx->N;
  const int nvec = n1 - n0 + 1;
  if (nvec > 32) return set_err(ctx, WTBG_ERR_UNSUPPORTED, "eigvecs: at most 32 vectors per launch");
  cudaStream_t s = ctx->stream;
  // tridiagonal eigenvectors of the requested range, recomputed by inverse iteration over
  // the whole clusters that contain n0-1 .. n1-1 (0-based)
  {
    const std::vector<int>& cs = ctx->csize_host;
    long long lead = n0 - 1;
    while (lead > 0 && cs[lead] == 0) --lead;
    long long end = n1 - 1;
    {
      long long l2 = end;
      while (l2 > 0 && cs[l2] == 0) --l2;
      end = l2 + cs[l2];
    }
    const long long M = end - lead;
    ENSURE(ctx->ws, (size_t)4 * 8 * n * M);
    ENSURE(ctx->zsel, (size_t)8 * n * nvec);
    ENSURE(ctx->tmp2, (size_t)8 * 8 * n);
    InvArgs a;
    a.d = ctx->d.as<double>();
    a.e = ctx->e.as<double>();
    a.n = n;
    a.lam = ctx->lam.as<double>();
    a.csize = ctx->csz.as<int>();
    a.m0 = lead;
    a.m1 = end;
    a.M = (int)M;
    a.ws = ctx->ws.as<double>();
    a.pert = DBL_EPSILON * std::max(ctx->tnorm, DBL_MIN);
    a.g = ctx->g.as<double2>();
    a.ng = ctx->ng;
    a.act = ctx->tmp2.as<double>();
    a.dtfull = 0;
    a.cpol = 0;
    a.zsel = ctx->zsel.as<double>();
    a.zs0 = n0 - 1;
    a.zs1 = n1 - 1;
    k_inviter<<<(int)((M + 63) / 64), 64, 0, s>>>(a); WTBG_COUNT(ctx, 1);
    CKL("k_inviter(eigvecs)");
  }
  const long long cnt = (long long)nvec * n;
  k_real_to_complex<<<(int)((cnt + 255) / 256), 256, 0, s>>>(ctx->zsel.as<double>(), d_out, cnt); WTBG_COUNT(ctx, 1);
  CKL("k_real_to_complex");
  if (ctx->tri_two) {
    if (int r = run_backtransform2(ctx, d_out, nvec)) return r;
    k_gauge_last<<<nvec, 256, 0, s>>>(d_out, n, nvec); WTBG_COUNT(ctx, 1);
    CKL("k_gauge_last");
    return 0;
  }
  const int nparts_max = (int)((n + BT_RB - 1) / BT_RB) + 1;
  ENSURE(ctx->tmp, (size_t)nparts_max * PB * (PB + 64) * 16 + PB * 64 * 16 + 1024);
  double2* part = ctx->tmp.as<double2>();
  double2* Y = part + (size_t)nparts_max * PB * (PB + 64);
  const size_t shb = (size_t)PB * (PB + 64) * 16;
  CK(cudaFuncSetAttribute(k_bt_gram, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shb));
  // panels in reverse order: Q X = P_0 (P_1 (... (P_last X)))
  const long long npan = (n - 1 + PB - 1) / PB;
  for (long long pnl = npan - 1; pnl >= 0; --pnl) {
    const int j0 = (int)(pnl * PB);
    const int jb = (int)std::min<long long>(PB, n - 1 - j0);
    const int nrows = (int)(n - j0 - 1);
    const int nparts = (nrows + BT_RB - 1) / BT_RB;
    k_bt_gram<<<nparts, BT_RB, shb, s>>>(ctx->H.as<double2>(), n, j0, jb, d_out, nvec, part); WTBG_COUNT(ctx, 1);
    k_bt_tmat<<<1, 256, 0, s>>>(part, nparts, jb, nvec, ctx->tau.as<double2>(), j0, Y); WTBG_COUNT(ctx, 1);
    k_bt_apply<<<(nrows + 255) / 256, 256, 0, s>>>(ctx->H.as<double2>(), n, j0, jb, d_out, nvec, Y); WTBG_COUNT(ctx, 1);
  }
  CKL("back-transform");
  k_gauge_last<<<nvec, 256, 0, s>>>(d_out, n, nvec); WTBG_COUNT(ctx, 1);
  CKL("k_gauge_last");
  return 0;
}
