// Kernel (a): Wannier Fourier sum H(k) = sum_R e^{i k.R} H(R)/deg(R) - E_F and the per-k
// Hermitian eigensolver, one CTA per k-point; plus the velocity matrices dH/dk_alpha
// and their band matrix elements (optsp), and the single-particle table.
//
// Reference: eigsys (subroutines/hamiltonian_tb.f90:2-137), band selection
// (subprograms/bse_solver-tool-diel.f90:257-313), hlm/optsp (subroutines/optics.f90:1-156),
// vecres + Bubblem (bse_solver-tool-diel.f90:379-402, general_subs.f90:405-440).
//
// Numerics that follow the reference exactly:
//   * the phase k.R is evaluated in double in the reference's order and rounded to
//     float32 before exp() (cmplx(0.0, x) without KIND, hamiltonian_tb.f90:64-66);
//   * E_F enters as float32 (fermilvl, hamiltonian_tb.f90:383);
//   * ZHEEV('V','Lower') reads the lower triangle and the real part of the diagonal, and
//     its eigenvectors have a real first component: the matrix is built from its lower
//     triangle and every eigenvector is rotated so that component 1 is real and >= 0
//     (the sign is irrelevant for every output of the path);
//   * the velocity prefactor i*R_alpha is float32-rounded (optics.f90:43-47) and the
//     optsp scale is Re(1/(E_c - E_v + i*float32(eta))) (REAL factor, optics.f90:114,148).
// The eigensolver is cyclic complex Jacobi in FP64 with a round-robin parallel ordering
// (w/2 disjoint rotations per step), converged to a relative threshold; it has an
// iteration cap and reports non-convergence per k instead of spinning.
#include <cfloat>
#include <cub/cub.cuh>

#include "common.cuh"

#include <algorithm>

namespace {

constexpr int kBandsThreads = 256;
constexpr int kMaxSweeps = 60;

struct Rot {
  int p, q, active, pad;
  double cs, sn, ex, ey, ap, aq;
};

__device__ __forceinline__ double2 phase_of(double kx, double ky, double kz, const double* R) {
  // (kx*Rx + ky*Ry) + kz*Rz, each product and sum rounded separately (no contraction)
  double kr = __dadd_rn(__dadd_rn(__dmul_rn(kx, R[0]), __dmul_rn(ky, R[1])), __dmul_rn(kz, R[2]));
  float kr32 = __double2float_rn(kr);
  double s, c;
  sincos((double)kr32, &s, &c);
  return make_double2(c, s);
}

struct BandsArgs {
  const double2* HR;
  const double* Rcart;
  const double* invdeg;
  int nvec, w;
  const double* kpt;
  int nk;
  double ef32, scs;
  int nv, nc;
  double* eig;     // [nk][nb]
  double2* U;      // [nk][nb][w]
  int* nocp;       // [nk]
  int* kstat;      // [nk]
  int all;         // 1: every band (eigsys as the band and DOS tools call it), nb = w
  const float* Hk; // precision form: H(k) from the tensor-core Fourier sum, [2 w^2][nk] (Re, Im)
  unsigned char* gwork;   // large models: per-CTA work areas in global memory (else shared memory)
  long long gstride;      // bytes per CTA work area
};

// One k-point per iteration of the loop k = k0, k0 + kstride, ... (shared-memory work area
// smem, sized by bands_smem for this model).
__device__ __forceinline__ void bands_body(const BandsArgs& a, int k0, int kstride, unsigned char* smem) {
  const int w = a.w, nvec = a.nvec, tid = threadIdx.x, bs = blockDim.x;
  const int ww = w * w;
  const int m2 = w + (w & 1);
  const int npair = m2 / 2;
  double2* ph = reinterpret_cast<double2*>(smem);
  double2* A = ph + nvec;
  double2* V = A + ww;
  Rot* rot = reinterpret_cast<Rot*>(V + ww);
  double* lam = reinterpret_cast<double*>(rot + npair);
  int* perm = reinterpret_cast<int*>(lam + w);
  double* red = reinterpret_cast<double*>(perm + w + (w & 1));  // kBandsThreads/32 doubles
  __shared__ int s_rotated;
  __shared__ double s_tolabs;
  __shared__ int s_nocp, s_stat;

  for (int k = k0; k < a.nk; k += kstride) {
    const double kx = a.kpt[3 * k], ky = a.kpt[3 * k + 1], kz = a.kpt[3 * k + 2];
    for (int R = tid; R < nvec; R += bs) ph[R] = phase_of(kx, ky, kz, a.Rcart + 3 * R);
    __syncthreads();
    // Fourier sum on the lower triangle (ZHEEV 'L' reads nothing else), R in file order
    double fro = 0.0;
    for (int el = tid; el < ww; el += bs) {
      const int m = el % w, n = el / w;
      double2 acc = make_double2(0.0, 0.0);
      if (m >= n && a.Hk) {
        acc = make_double2((double)a.Hk[(size_t)el * a.nk + k], (double)a.Hk[(size_t)(ww + el) * a.nk + k]);
        if (m == n) acc = make_double2(acc.x + (-a.ef32), 0.0);
        fro += (m == n ? 1.0 : 2.0) * (acc.x * acc.x + acc.y * acc.y);
      } else if (m >= n) {
        const double2* hp = a.HR + el;
        for (int R = 0; R < nvec; ++R) {
          double2 t = cmul(ph[R], hp[(size_t)R * ww]);
          acc = cadd(acc, cscale(t, a.invdeg[R]));
        }
        if (m == n) acc = make_double2(acc.x + (-a.ef32), 0.0);
        fro += (m == n ? 1.0 : 2.0) * (acc.x * acc.x + acc.y * acc.y);
      }
      A[el] = acc;
      V[el] = make_double2(m == n ? 1.0 : 0.0, 0.0);
    }
    // block reduction of the Frobenius norm
    for (int o = 16; o > 0; o >>= 1) fro += __shfl_xor_sync(0xffffffffu, fro, o);
    if ((tid & 31) == 0) red[tid >> 5] = fro;
    __syncthreads();
    if (tid == 0) {
      double s = 0.0;
      for (int i = 0; i < bs / 32; ++i) s += red[i];
      s_tolabs = DBL_EPSILON * 1e-2 * sqrt(s);
      s_stat = 1;  // not converged until proven
    }
    for (int el = tid; el < ww; el += bs) {
      const int m = el % w, n = el / w;
      if (m < n) A[el] = cconj(A[n + m * w]);
    }
    __syncthreads();

    for (int sweep = 0; sweep < kMaxSweeps; ++sweep) {
      if (tid == 0) s_rotated = 0;
      __syncthreads();
      for (int r = 0; r < m2 - 1; ++r) {
        if (tid < npair) {
          const int t = tid;
          int p = (t == 0) ? (m2 - 1) : ((r + t - 1) % (m2 - 1));
          int q = (r + (m2 - 1 - t) - 1) % (m2 - 1);
          Rot ro;
          ro.active = 0;
          if (p > q) { int x = p; p = q; q = x; }
          ro.p = p;
          ro.q = q;
          if (q < w) {
            const double aa = A[p + p * w].x, bb = A[q + q * w].x;
            const double2 c = A[p + q * w];
            const double ac = hypot(c.x, c.y);
            const double thr = fmax(0.5 * DBL_EPSILON * sqrt(fabs(aa * bb)), s_tolabs);
            if (ac > thr && ac > 0.0) {
              const double zeta = (bb - aa) / (2.0 * ac);
              double tt;
              if (fabs(zeta) > 1e150) tt = 0.5 / zeta;
              else tt = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
              const double cs = 1.0 / sqrt(1.0 + tt * tt);
              ro.cs = cs;
              ro.sn = tt * cs;
              ro.ex = c.x / ac;
              ro.ey = c.y / ac;
              ro.ap = aa - tt * ac;
              ro.aq = bb + tt * ac;
              ro.active = 1;
              s_rotated = 1;
            }
          }
          rot[t] = ro;
        }
        __syncthreads();
        // rows: A <- J^H A
        for (int it = tid; it < npair * w; it += bs) {
          const Rot& ro = rot[it / w];
          if (!ro.active) continue;
          const int col = it % w;
          const double2 e = make_double2(ro.ex, ro.ey);
          const double2 rp = A[ro.p + col * w], rq = A[ro.q + col * w];
          A[ro.p + col * w] = csub(cscale(rp, ro.cs), cscale(cmul(e, rq), ro.sn));
          A[ro.q + col * w] = cadd(cscale(cmulc(e, rp), ro.sn), cscale(rq, ro.cs));
        }
        __syncthreads();
        // columns: A <- A J, V <- V J
        for (int it = tid; it < npair * w; it += bs) {
          const Rot& ro = rot[it / w];
          if (!ro.active) continue;
          const int row = it % w;
          const double2 e = make_double2(ro.ex, ro.ey);
          double2 cp = A[row + ro.p * w], cq = A[row + ro.q * w];
          A[row + ro.p * w] = csub(cscale(cp, ro.cs), cscale(cmulc(e, cq), ro.sn));
          A[row + ro.q * w] = cadd(cscale(cmul(e, cp), ro.sn), cscale(cq, ro.cs));
          cp = V[row + ro.p * w];
          cq = V[row + ro.q * w];
          V[row + ro.p * w] = csub(cscale(cp, ro.cs), cscale(cmulc(e, cq), ro.sn));
          V[row + ro.q * w] = cadd(cscale(cmul(e, cp), ro.sn), cscale(cq, ro.cs));
        }
        __syncthreads();
        if (tid < npair) {
          const Rot& ro = rot[tid];
          if (ro.active) {
            A[ro.p + ro.q * w] = make_double2(0.0, 0.0);
            A[ro.q + ro.p * w] = make_double2(0.0, 0.0);
            A[ro.p + ro.p * w] = make_double2(ro.ap, 0.0);
            A[ro.q + ro.q * w] = make_double2(ro.aq, 0.0);
          }
        }
        __syncthreads();
      }
      const int any = s_rotated;
      __syncthreads();
      if (!any) {
        if (tid == 0) s_stat = 0;
        break;
      }
    }
    __syncthreads();
    // ascending order (ties by index), nocp, gauge
    if (tid < w) lam[tid] = A[tid + tid * w].x;
    __syncthreads();
    if (tid < w) {
      const double lj = lam[tid];
      int rank = 0;
      for (int i = 0; i < w; ++i) {
        const double li = lam[i];
        rank += (li < lj || (li == lj && i < tid)) ? 1 : 0;
      }
      perm[rank] = tid;
    }
    __syncthreads();
    if (tid == 0) {
      int nocp = -1;
      for (int i = 0; i < w; ++i) {
        if (lam[perm[i]] > 0.0) { nocp = i; break; }
      }
      int st = s_stat;
      if (st == 0 && !a.all) {
        if (nocp < 0) st = 2;
        else if (a.nv > nocp || a.nc > w - nocp) st = 3;
      }
      s_stat = st;
      s_nocp = nocp < 0 ? w : nocp;
      a.kstat[k] = st;
      a.nocp[k] = s_nocp;
    }
    __syncthreads();
    const int nb = a.all ? w : a.nv + a.nc;
    if (s_stat == 0) {
      const int nocp = s_nocp;
      const int off = a.all ? 0 : nocp - a.nv;   // all: band sel itself, scissors from nocp on
      for (int it = tid; it < nb * w; it += bs) {
        const int sel = it / w, m = it % w;
        const int src = perm[off + sel];
        const double2 v0 = V[src * w];
        const double r = hypot(v0.x, v0.y);
        double2 g = make_double2(1.0, 0.0);
        if (r > 0.0) g = make_double2(v0.x / r, -v0.y / r);
        a.U[((size_t)k * nb + sel) * w + m] = cmul(V[m + src * w], g);
        if (m == 0) a.eig[(size_t)k * nb + sel] = lam[src] + (sel >= (a.all ? nocp : a.nv) ? a.scs : 0.0);
      }
    }
    __syncthreads();
  }
}

// Precision form of the Fourier sum H(k) = sum_R e^{i k.R} H(R) / deg(R) as one real GEMM
// over all k: A rows k = [Re P | Im P] with P(k,R) = phase / deg, B rows (Re out) [Re H | -Im H]
// and (Im out) [Im H | Re H] per matrix element; segments padded to S (a multiple of 8).
__global__ void k_hk_opA(const double* kpt, const double* Rcart, const double* invdeg, int nvec, int S,
                         __nv_bfloat16* A3) {
  const int k = blockIdx.x;
  __nv_bfloat16* row = A3 + (size_t)k * 6 * S;
  for (int R = threadIdx.x; R < S; R += blockDim.x) {
    double2 p = make_double2(0, 0);
    if (R < nvec) p = cscale(phase_of(kpt[3 * k], kpt[3 * k + 1], kpt[3 * k + 2], Rcart + 3 * R), invdeg[R]);
    put_split_row(row, 2 * S, R, p.x, true);
    put_split_row(row, 2 * S, S + R, p.y, true);
  }
}

__global__ void k_hk_opB(const double2* HR, int nvec, int ww, int S, __nv_bfloat16* B3) {
  const int j = blockIdx.x, el = j % ww;
  const bool im = j >= ww;
  __nv_bfloat16* row = B3 + (size_t)j * 6 * S;
  for (int R = threadIdx.x; R < S; R += blockDim.x) {
    double x = 0.0, y = 0.0;
    if (R < nvec) {
      const double2 h = HR[(size_t)R * ww + el];
      x = im ? h.y : h.x;
      y = im ? h.x : -h.y;
    }
    put_split_row(row, 2 * S, R, x, false);
    put_split_row(row, 2 * S, S + R, y, false);
  }
}

// work area of this CTA: dynamic shared memory, or its slice of the global work buffer when
// the model's matrices exceed the shared-memory budget (w above ~70)
__device__ __forceinline__ unsigned char* work_base(unsigned char* smem, unsigned char* gwork, long long gstride) {
  return gwork ? gwork + (size_t)blockIdx.x * (size_t)gstride : smem;
}

__global__ void __launch_bounds__(kBandsThreads) k_bands(BandsArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  bands_body(a, blockIdx.x, gridDim.x, work_base(smem, a.gwork, a.gstride));
}

// Persistent ragged batch: every (model, k) item of several models (different w, nvec and
// meshes) in one launch. Items are ordered by decreasing w; each CTA takes the next item
// from a global counter, so the expensive large-w items start first.
__global__ void __launch_bounds__(kBandsThreads) k_bands_batch(const BandsArgs* mods, const int* item_mod,
                                                               const int* item_k, int nitems, int* counter) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_item;
  while (true) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= nitems) break;
    const BandsArgs a = mods[item_mod[it]];
    const int k = item_k[it];
    bands_body(a, k, a.nk, work_base(smem, a.gwork, a.gstride));
  }
}

// ---------------------------------------------------------------------------------------
struct VelArgs {
  const double2* HR;
  const double* Rcart;
  const double* Rf32;
  const double* invdeg;
  const int* isR0;
  int nvec, w;
  const double* kpt;
  int nk, nv, nc;
  const double* eig;
  const double2* U;
  double eta32;
  double inv_sqrt2_f32;
  double2* h;      // [5][N]
  long long N;
  unsigned char* gwork;
  long long gstride;
};

__global__ void __launch_bounds__(kBandsThreads) k_velocity(VelArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int w = a.w, nvec = a.nvec, tid = threadIdx.x, bs = blockDim.x;
  const int ww = w * w, nb = a.nv + a.nc;
  double2* ph = reinterpret_cast<double2*>(work_base(smem, a.gwork, a.gstride));
  double2* HX = ph + nvec;          // 3 matrices, column-major
  double2* Us = HX + 3 * ww;        // nb x w
  double2* T = Us + nb * w;         // [3][nv][w] = h_alpha * u_v
  for (int k = blockIdx.x; k < a.nk; k += gridDim.x) {
    const double kx = a.kpt[3 * k], ky = a.kpt[3 * k + 1], kz = a.kpt[3 * k + 2];
    for (int R = tid; R < nvec; R += bs) ph[R] = phase_of(kx, ky, kz, a.Rcart + 3 * R);
    for (int it = tid; it < nb * w; it += bs) Us[it] = a.U[(size_t)k * nb * w + it];
    __syncthreads();
    for (int el = tid; el < ww; el += bs) {
      const int m = el % w, n = el / w;
      double2 acc[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
      const double2* hp = a.HR + el;
      for (int R = 0; R < nvec; ++R) {
        if (m == n && a.isR0[R]) continue;   // R=0 diagonal zeroed (optics.f90:59-68)
        const double2 hr = hp[(size_t)R * ww];
        const double2 p = ph[R];
        const double inv = a.invdeg[R];
#pragma unroll
        for (int al = 0; al < 3; ++al) {
          const double ra = a.Rf32[3 * R + al];
          const double2 pre = make_double2(-ra * p.y, ra * p.x);   // (i*R_alpha) * phase
          acc[al] = cadd(acc[al], cscale(cmul(pre, hr), inv));
        }
      }
      HX[el] = acc[0];
      HX[ww + el] = acc[1];
      HX[2 * ww + el] = acc[2];
    }
    __syncthreads();
    // T[al][v][m] = sum_n H_al[m,n] u_v[n]   (matvec, general_subs.f90:132-160)
    for (int it = tid; it < 3 * a.nv * w; it += bs) {
      const int m = it % w, v = (it / w) % a.nv, al = it / (w * a.nv);
      const double2* Hm = HX + al * ww;
      const double2* uv = Us + v * w;
      double2 acc = make_double2(0, 0);
      for (int n = 0; n < w; ++n) acc = cadd(acc, cmul(Hm[m + n * w], uv[n]));
      T[it] = acc;
    }
    __syncthreads();
    // h = Re(1/(dE + i eta)) * <c| H_al |v>   for the (c, v) pairs of this k
    for (int it = tid; it < a.nc * a.nv; it += bs) {
      const int c = it / a.nv, v = it % a.nv;
      const double2* uc = Us + (a.nv + c) * w;
      const double de = a.eig[(size_t)k * nb + a.nv + c] - a.eig[(size_t)k * nb + v];
      const double factor = de / (de * de + a.eta32 * a.eta32);
      double2 hr[3];
#pragma unroll
      for (int al = 0; al < 3; ++al) {
        const double2* t = T + (al * a.nv + v) * w;
        double2 acc = make_double2(0, 0);
        for (int m = 0; m < w; ++m) acc = cadd(acc, cmulc(uc[m], t[m]));
        hr[al] = cscale(acc, factor);
      }
      const long long i = (long long)k * a.nc * a.nv + c * a.nv + v;
      a.h[i] = hr[0];
      a.h[a.N + i] = hr[1];
      a.h[2 * a.N + i] = hr[2];
      const double s = a.inv_sqrt2_f32;
      a.h[3 * a.N + i] = cscale(make_double2(hr[0].x - hr[1].y, hr[0].y + hr[1].x), s);
      a.h[4 * a.N + i] = cscale(make_double2(hr[0].x + hr[1].y, hr[0].y - hr[1].x), s);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------
// Berry curvature per k (berryct2, berry_curvature_subs.f90:1-128):
//   b_ab = sum_{n <= nocp < i} -2 v_a(n,i) conj(v_b(n,i)) / ((E_n - E_i)^2 + gamma^2),
//   v_a(n,i) = <n| dH/dk_a |i>  (hlm, optics.f90:1-97, as in k_velocity),
// pairs with |E_i - E_n| < degtol skipped. One CTA per k; the three dH/dk matrices are built
// in shared memory and overwritten by T_a = dH/dk_a U (unoccupied columns); the pair sums are
// reduced over the block. out[c * nk + k] = Im b_c, c = xx, xy, xz, yy, yz, zz.
// dH/dk_a of hlm (optics.f90:1-97) at one k into shared memory: HX = three column-major w x w
// matrices, ph = the nvec phases (work area). Ends with a block barrier.
__device__ void hlm_smem(const double2* HR, const double* Rcart, const double* Rf32, const double* invdeg,
                         const int* isR0, int nvec, int w, double kx, double ky, double kz, double2* ph, double2* HX) {
  const int tid = threadIdx.x, bs = blockDim.x, ww = w * w;
  for (int R = tid; R < nvec; R += bs) ph[R] = phase_of(kx, ky, kz, Rcart + 3 * R);
  __syncthreads();
  for (int el = tid; el < ww; el += bs) {
    const int m = el % w, n = el / w;
    double2 acc[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    const double2* hp = HR + el;
    for (int R = 0; R < nvec; ++R) {
      if (m == n && isR0[R]) continue;   // R=0 diagonal zeroed (optics.f90:59-68)
      const double2 hr = hp[(size_t)R * ww];
      const double2 p = ph[R];
      const double inv = invdeg[R];
#pragma unroll
      for (int al = 0; al < 3; ++al) {
        const double ra = Rf32[3 * R + al];
        const double2 pre = make_double2(-ra * p.y, ra * p.x);   // (i*R_alpha) * phase
        acc[al] = cadd(acc[al], cscale(cmul(pre, hr), inv));
      }
    }
    HX[el] = acc[0];
    HX[ww + el] = acc[1];
    HX[2 * ww + el] = acc[2];
  }
  __syncthreads();
}

struct BerryArgs {
  const double2* HR;
  const double* Rcart;
  const double* Rf32;
  const double* invdeg;
  const int* isR0;
  int nvec, w, nk;
  const double* kpt;
  const double* eig;    // [nk][w]
  const double2* U;     // [nk][w][w], band-major
  const int* nocp;      // [nk]
  double gamma2, degtol;
  double* out;          // [6][nk]
  unsigned char* gwork;
  long long gstride;
};

__global__ void __launch_bounds__(kBandsThreads) k_berry(BerryArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int w = a.w, nvec = a.nvec, tid = threadIdx.x, bs = blockDim.x;
  const int ww = w * w;
  double2* ph = reinterpret_cast<double2*>(work_base(smem, a.gwork, a.gstride));
  double2* HX = ph + nvec;      // 3 matrices, column-major; then T_a
  double2* Us = HX + 3 * ww;    // U[band][m]
  double2* tmp = Us + ww;       // one T_a before it replaces dH/dk_a
  __shared__ double red[kBandsThreads / 32][12];
  for (int k = blockIdx.x; k < a.nk; k += gridDim.x) {
    const double kx = a.kpt[3 * k], ky = a.kpt[3 * k + 1], kz = a.kpt[3 * k + 2];
    const int nocp = a.nocp[k];
    for (int it = tid; it < ww; it += bs) Us[it] = a.U[(size_t)k * ww + it];
    hlm_smem(a.HR, a.Rcart, a.Rf32, a.invdeg, a.isR0, nvec, w, kx, ky, kz, ph, HX);
    // T_a[m][i] = sum_l H_a[m][l] u_i[l] for the unoccupied bands i (matvec, general_subs.f90:132-160)
    for (int al = 0; al < 3; ++al) {
      double2* Ha = HX + al * ww;
      for (int it = tid; it < w * (w - nocp); it += bs) {
        const int m = it % w, i = nocp + it / w;
        const double2* ui = Us + i * w;
        double2 acc = make_double2(0, 0);
        for (int l = 0; l < w; ++l) acc = cadd(acc, cmul(Ha[m + l * w], ui[l]));
        tmp[m + i * w] = acc;
      }
      __syncthreads();
      for (int it = tid; it < w * (w - nocp); it += bs) {
        const int m = it % w, i = nocp + it / w;
        Ha[m + i * w] = tmp[m + i * w];
      }
      __syncthreads();
    }
    double2 b[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) b[c] = make_double2(0, 0);
    const int nun = w - nocp;
    for (int it = tid; it < nocp * nun; it += bs) {
      const int n = it / nun, i = nocp + it % nun;
      const double en = a.eig[(size_t)k * w + n], ei = a.eig[(size_t)k * w + i];
      if (fabs(ei - en) < a.degtol) continue;
      const double2* un = Us + n * w;
      double2 v[3];
#pragma unroll
      for (int al = 0; al < 3; ++al) {
        const double2* t = HX + al * ww + i * w;
        double2 acc = make_double2(0, 0);
        for (int m = 0; m < w; ++m) acc = cadd(acc, cmulc(un[m], t[m]));   // prodintsq(conj(u_n), T u_i)
        v[al] = acc;
      }
      const double aux = (en - ei) * (en - ei) + a.gamma2;
      const int pa[6] = {0, 0, 0, 1, 1, 2}, pb[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        const double2 pr = cmul(v[pa[c]], cconj(v[pb[c]]));
        b[c] = cadd(b[c], make_double2(-2.0 * (pr.x / aux), -2.0 * (pr.y / aux)));
      }
    }
    // block reduction of the six sums (only the imaginary parts are kept)
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      double x = b[c].y;
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if ((tid & 31) == 0) red[tid >> 5][c] = x;
    }
    __syncthreads();
    if (tid < 6) {
      double s = 0.0;
      for (int q = 0; q < bs / 32; ++q) s += red[q][tid];
      a.out[(size_t)tid * a.nk + k] = s;
    }
    __syncthreads();
  }
}

// Single-particle optical activity over the BZ (spoptpolbz, sp_opt_bz-tool.f90:81-175): per k,
// the pairs (c, v) with c = nocp_k .. nocp_k + nc - 1 (outer) and v = nocp_k - nv .. nocp_1 - 1
// (inner; the reference bounds v by the FIRST k-point's nocp), the first nc * nv of them;
// h_a = <c|dH/dk_a|v> / (f32(E_c - E_v) + i f32(sme)) (optspbz, optics.f90:246-300, divided by a
// default-kind complex), and out[c * nk + k] = sum |h_x|^2, |h_y|^2, |h_z|^2,
// |norm (h_x + i h_y)|^2, |norm (h_x - i h_y)|^2 with norm = f32(1/sqrt 2). kstat = 4 where
// fewer than nc * nv pairs exist (the reference's pair table is then undefined).
struct OptBzArgs {
  const double2* HR;
  const double* Rcart;
  const double* Rf32;
  const double* invdeg;
  const int* isR0;
  int nvec, w, nk, nv, nc;
  const double* kpt;
  const double* eig;    // [nk][w]
  const double2* U;     // [nk][w][w]
  const int* nocp;      // [nk]
  double sme32, norm32;
  double* out;          // [5][nk]
  int* kstat;
  unsigned char* gwork;
  long long gstride;
};

__global__ void __launch_bounds__(kBandsThreads) k_optbz(OptBzArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int w = a.w, nvec = a.nvec, tid = threadIdx.x, bs = blockDim.x;
  const int ww = w * w;
  double2* ph = reinterpret_cast<double2*>(work_base(smem, a.gwork, a.gstride));
  double2* HX = ph + nvec;
  double2* Us = HX + 3 * ww;
  __shared__ double red[kBandsThreads / 32][5];
  const int nocp1 = a.nocp[0];
  for (int k = blockIdx.x; k < a.nk; k += gridDim.x) {
    const double kx = a.kpt[3 * k], ky = a.kpt[3 * k + 1], kz = a.kpt[3 * k + 2];
    const int nocp = a.nocp[k];
    const int vlo = nocp - a.nv, nvv = max(0, nocp1 - vlo);
    const int npair_all = a.nc * nvv, npair = min(npair_all, a.nc * a.nv);
    for (int it = tid; it < ww; it += bs) Us[it] = a.U[(size_t)k * ww + it];
    hlm_smem(a.HR, a.Rcart, a.Rf32, a.invdeg, a.isR0, nvec, w, kx, ky, kz, ph, HX);
    double s[5] = {0, 0, 0, 0, 0};
    for (int p = tid; p < npair; p += bs) {
      const int c = nocp + p / nvv, v = vlo + p % nvv;
      if (c >= w || v < 0) continue;
      const double2* uc = Us + c * w;
      const double2* uv = Us + v * w;
      double2 h[3];
#pragma unroll
      for (int al = 0; al < 3; ++al) {
        const double2* Ha = HX + al * ww;
        double2 acc = make_double2(0, 0);
        for (int m = 0; m < w; ++m) {
          double2 t = make_double2(0, 0);
          for (int l = 0; l < w; ++l) t = cadd(t, cmul(Ha[m + l * w], uv[l]));
          acc = cadd(acc, cmulc(uc[m], t));
        }
        h[al] = acc;
      }
      const double dr = (double)(float)(a.eig[(size_t)k * w + c] - a.eig[(size_t)k * w + v]);
      const double den = dr * dr + a.sme32 * a.sme32;
      const double2 sp = make_double2(h[0].x - h[1].y, h[0].y + h[1].x);   // h_x + i h_y
      const double2 sm = make_double2(h[0].x + h[1].y, h[0].y - h[1].x);   // h_x - i h_y
      s[0] += (h[0].x * h[0].x + h[0].y * h[0].y) / den;
      s[1] += (h[1].x * h[1].x + h[1].y * h[1].y) / den;
      s[2] += (h[2].x * h[2].x + h[2].y * h[2].y) / den;
      s[3] += a.norm32 * a.norm32 * (sp.x * sp.x + sp.y * sp.y) / den;
      s[4] += a.norm32 * a.norm32 * (sm.x * sm.x + sm.y * sm.y) / den;
    }
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      double x = s[c];
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if ((tid & 31) == 0) red[tid >> 5][c] = x;
    }
    __syncthreads();
    if (tid < 5) {
      double t = 0.0;
      for (int q = 0; q < bs / 32; ++q) t += red[q][tid];
      a.out[(size_t)tid * a.nk + k] = t;
    }
    if (tid == 0 && npair_all < a.nc * a.nv) a.kstat[k] = 4;
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------
// vecres rows (bse_solver-tool-diel.f90:379-393); key = column 7 (float32 dE)
__global__ void k_sp_rows(const double* kpt, const double* eig, const int* nocp, const double2* h, const double* fdeh,
                          int nk, int nv, int nc, long long N, float* rows, float* key, int* idx) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int ncv = nc * nv, nb = nc + nv;
  const int k = (int)(i / ncv), c = (int)((i % ncv) / nv), v = (int)(i % nv);
  const double2 hx = h[i], hy = h[N + i], hz = h[2 * N + i], hp = h[3 * N + i], hm = h[4 * N + i];
  float* r = rows + i * 15;
  r[0] = (float)kpt[3 * k];
  r[1] = (float)kpt[3 * k + 1];
  r[2] = (float)kpt[3 * k + 2];
  r[3] = (float)nocp[k];
  r[4] = (float)(nocp[k] - nv + (nv + c + 1));
  r[5] = (float)(nocp[k] - nv + (v + 1));
  r[6] = (float)(eig[(size_t)k * nb + nv + c] - eig[(size_t)k * nb + v]);
  if (fdeh == nullptr) {
    r[7] = (float)(hx.x * hx.x + hx.y * hx.y);
    r[8] = (float)(hy.x * hy.x + hy.y * hy.y);
    r[9] = (float)(hz.x * hz.x + hz.y * hz.y);
    r[10] = (float)(hx.x * hy.x + hx.y * hy.y);
    r[11] = (float)(hx.x * hz.x + hx.y * hz.y);
    r[12] = (float)(hy.x * hz.x + hy.y * hz.y);
    r[13] = (float)(hp.x * hp.x + hp.y * hp.y);
    r[14] = (float)(hm.x * hm.x + hm.y * hm.y);
  } else {   // temperature: the strengths times f_v - f_c (bse_solver-tool-diel-temp.f90:416-423)
    const double f = fdeh[i];
    r[7] = (float)((hx.x * hx.x + hx.y * hx.y) * f);
    r[8] = (float)((hy.x * hy.x + hy.y * hy.y) * f);
    r[9] = (float)((hz.x * hz.x + hz.y * hz.y) * f);
    r[10] = (float)((hx.x * hy.x + hx.y * hy.y) * f);
    r[11] = (float)((hx.x * hz.x + hx.y * hz.y) * f);
    r[12] = (float)((hy.x * hz.x + hy.y * hz.y) * f);
    r[13] = (float)((hp.x * hp.x + hp.y * hp.y) * f);
    r[14] = (float)((hm.x * hm.x + hm.y * hm.y) * f);
  }
  key[i] = r[6];
  idx[i] = (int)i;
}

__global__ void k_sp_gather(const float* rows, const int* order, long long N, float* out) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float* r = rows + (long long)order[i] * 15;
#pragma unroll
  for (int c = 0; c < 15; ++c) out[c * N + i] = r[c];
}

}  // namespace

// Work-area placement of the per-k kernels: the model's matrices go to dynamic shared memory
// when they fit the budget, else every CTA of a grid capped at 4 CTAs per SM gets a slice of
// ctx->gwork in global memory (L2-resident at these sizes) and loops over k.
constexpr size_t kSmemBudget = 200 * 1024;
static int place_work(wtbg_ctx* ctx, size_t bytes, long long nk, unsigned char** gwork, long long* gstride,
                      size_t* dyn, int* grid) {
  if (bytes <= kSmemBudget) {
    *gwork = nullptr;
    *gstride = 0;
    *dyn = bytes;
    *grid = (int)nk;
    return 0;
  }
  if (ctx->nsm <= 0) CK(cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, ctx->device));
  const long long g = std::min<long long>(nk, 4LL * ctx->nsm);
  const size_t stride = (bytes + 255) / 256 * 256;
  ENSURE(ctx->gwork, stride * (size_t)g);
  *gwork = ctx->gwork.as<unsigned char>();
  *gstride = (long long)stride;
  *dyn = 0;
  *grid = (int)g;
  return 0;
}

static size_t bands_smem(int w, int nvec) {
  const int ww = w * w, m2 = w + (w & 1);
  return (size_t)nvec * 16 + 2 * (size_t)ww * 16 + (size_t)(m2 / 2) * sizeof(Rot) + (size_t)w * 8 +
         (size_t)(w + (w & 1)) * 4 + 64 * 8;
}

// H(k) of every k of the mesh by the 3-term split-BF16 tensor-core GEMM (FP32 result
// [2 w^2][nk] in ctx->pHk)
static int run_precision_hk(wtbg_ctx* ctx, const double* kpt, int nk) {
  const int w = ctx->w, ww = w * w, nvec = ctx->nvec;
  const int S = (nvec + 7) / 8 * 8, K = 6 * S;
  ENSURE(ctx->pOpA, (size_t)nk * K * 2);
  ENSURE(ctx->pOpB, (size_t)2 * ww * K * 2);
  ENSURE(ctx->pHk, (size_t)2 * ww * nk * 4);
  ENSURE(ctx->pErr, 16);
  __nv_bfloat16* A3 = ctx->pOpA.as<__nv_bfloat16>();
  __nv_bfloat16* B3 = ctx->pOpB.as<__nv_bfloat16>();
  k_hk_opA<<<nk, 128, 0, ctx->stream>>>(kpt, ctx->Rcart.as<double>(), ctx->invdeg.as<double>(), nvec, S, A3);
  k_hk_opB<<<2 * ww, 128, 0, ctx->stream>>>(ctx->HR.as<double2>(), nvec, ww, S, B3);
  WTBG_COUNT(ctx, 2);
  CKL("k_hk_op");
  return gemm_bf16(ctx, ctx->pErr.as<int>(), A3, K, nk, K, B3, K, 2 * ww, ctx->pHk.as<float>(), nk, true);
}

int launch_bands(wtbg_ctx* ctx, bool q_mesh) {
  const int w = ctx->w;
  BandsArgs a;
  a.HR = ctx->HR.as<double2>();
  a.Rcart = ctx->Rcart.as<double>();
  a.invdeg = ctx->invdeg.as<double>();
  a.nvec = ctx->nvec;
  a.w = w;
  a.nk = ctx->nk;
  a.ef32 = (double)(float)ctx->efermi;
  a.scs = ctx->scs;
  a.nv = ctx->nv;
  a.nc = ctx->nc;
  if (q_mesh) {
    a.kpt = ctx->kptq.as<double>();
    a.eig = ctx->eigq.as<double>();
    a.U = ctx->Uq.as<double2>();
    a.nocp = ctx->nocpq.as<int>();
  } else {
    a.kpt = ctx->kpt.as<double>();
    a.eig = ctx->eig.as<double>();
    a.U = ctx->U.as<double2>();
    a.nocp = ctx->nocp.as<int>();
  }
  a.kstat = ctx->kstat.as<int>();
  a.all = 0;
  a.Hk = nullptr;
  if (ctx->prec == 1) {
    if (int r = run_precision_hk(ctx, a.kpt, ctx->nk)) return r;
    a.Hk = ctx->pHk.as<float>();
  }
  size_t smem = 0;
  int grid = 0;
  if (int r = place_work(ctx, bands_smem(w, ctx->nvec), ctx->nk, &a.gwork, &a.gstride, &smem, &grid)) return r;
  CK(cudaFuncSetAttribute(k_bands, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_bands<<<grid, kBandsThreads, smem, ctx->stream>>>(a); WTBG_COUNT(ctx, 1);
  CKL("k_bands");
  return 0;
}

// Bands of several models on one device in one persistent launch (the contexts share a
// device; the launch goes on the first context's stream). Each context gets its own k-mesh
// bands exactly as launch_bands would produce them.
int launch_bands_batch(wtbg_ctx* const* ctxs, int nmod) {
  wtbg_ctx* c0 = ctxs[0];
  wtbg_ctx* ctx = c0;   // errors and scratch on the first context
  std::vector<BandsArgs> mods(nmod);
  std::vector<std::pair<int, int>> order;   // (w, model)
  size_t smem = 0;
  long long nitems = 0;
  for (int m = 0; m < nmod; ++m) {
    wtbg_ctx* cm = ctxs[m];
    BandsArgs& a = mods[m];
    a.HR = cm->HR.as<double2>();
    a.Rcart = cm->Rcart.as<double>();
    a.invdeg = cm->invdeg.as<double>();
    a.nvec = cm->nvec;
    a.w = cm->w;
    a.nk = cm->nk;
    a.ef32 = (double)(float)cm->efermi;
    a.scs = cm->scs;
    a.nv = cm->nv;
    a.nc = cm->nc;
    a.kpt = cm->kpt.as<double>();
    a.eig = cm->eig.as<double>();
    a.U = cm->U.as<double2>();
    a.nocp = cm->nocp.as<int>();
    a.kstat = cm->kstat.as<int>();
    a.all = 0;
    a.Hk = nullptr;   // the batch runs the FP64 form
    smem = std::max(smem, bands_smem(cm->w, cm->nvec));
    order.push_back({cm->w, m});
    nitems += cm->nk;
  }
  std::stable_sort(order.begin(), order.end(), [](const std::pair<int, int>& x, const std::pair<int, int>& y) {
    return x.first > y.first;
  });
  std::vector<int> im, ik;
  im.reserve(nitems);
  ik.reserve(nitems);
  for (auto& o : order)
    for (int k = 0; k < ctxs[o.second]->nk; ++k) {
      im.push_back(o.second);
      ik.push_back(k);
    }
  const size_t b_mod = (size_t)nmod * sizeof(BandsArgs), b_it = (size_t)nitems * 4;
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  ENSURE(c0->tmp, up(b_mod) + 2 * up(b_it) + 256);
  char* base = c0->tmp.as<char>();
  BandsArgs* d_mod = reinterpret_cast<BandsArgs*>(base);
  int* d_im = reinterpret_cast<int*>(base + up(b_mod));
  int* d_ik = reinterpret_cast<int*>(base + up(b_mod) + up(b_it));
  int* d_cnt = reinterpret_cast<int*>(base + up(b_mod) + 2 * up(b_it));
  cudaStream_t s = c0->stream;
  CK(cudaMemcpyAsync(d_mod, mods.data(), b_mod, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_im, im.data(), b_it, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_ik, ik.data(), b_it, cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(d_cnt, 0, 4, s));
  int dev = 0, nsm = 148, per = 1;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  if (smem > kSmemBudget) {
    // a model too large for shared memory: every CTA works in its slice of global memory
    const long long g = std::min<long long>(nitems, 4LL * nsm);
    const size_t stride = (smem + 255) / 256 * 256;
    ENSURE(c0->gwork, stride * (size_t)g);
    for (auto& a : mods) {
      a.gwork = c0->gwork.as<unsigned char>();
      a.gstride = (long long)stride;
    }
    CK(cudaMemcpyAsync(d_mod, mods.data(), b_mod, cudaMemcpyHostToDevice, s));
    smem = 0;
    per = 4;
  }
  CK(cudaFuncSetAttribute(k_bands_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  if (smem > 0) CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_bands_batch, kBandsThreads, smem));
  const int grid = (int)std::min<long long>(nitems, (long long)nsm * std::max(1, per));
  k_bands_batch<<<grid, kBandsThreads, smem, s>>>(d_mod, d_im, d_ik, (int)nitems, d_cnt);
  WTBG_COUNT(c0, 1);
  {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c0, e, "k_bands_batch");
  }
  return 0;
}

// every band of every k (eigsys of the band and DOS tools): eig [nk][w], U [nk][w][w]
int launch_eigsys_all(wtbg_ctx* ctx, int nk, const double* d_kpt, double* d_eig, double2* d_U, int* d_nocp,
                      int* d_kstat) {
  const int w = ctx->w;
  BandsArgs a;
  a.HR = ctx->HR.as<double2>();
  a.Rcart = ctx->Rcart.as<double>();
  a.invdeg = ctx->invdeg.as<double>();
  a.nvec = ctx->nvec;
  a.w = w;
  a.nk = nk;
  a.ef32 = (double)(float)ctx->efermi;
  a.scs = ctx->scs;
  a.nv = 0;
  a.nc = w;
  a.kpt = d_kpt;
  a.eig = d_eig;
  a.U = d_U;
  a.nocp = d_nocp;
  a.kstat = d_kstat;
  a.all = 1;
  a.Hk = nullptr;   // the band and DOS tools run the FP64 form
  size_t smem = 0;
  int grid = 0;
  if (int r = place_work(ctx, bands_smem(w, ctx->nvec), nk, &a.gwork, &a.gstride, &smem, &grid)) return r;
  CK(cudaFuncSetAttribute(k_bands, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_bands<<<grid, kBandsThreads, smem, ctx->stream>>>(a); WTBG_COUNT(ctx, 1);
  CKL("k_bands(all)");
  return 0;
}

int launch_velocity(wtbg_ctx* ctx, double eta32) {
  const int w = ctx->w, nb = ctx->nv + ctx->nc;
  VelArgs a;
  a.HR = ctx->HR.as<double2>();
  a.Rcart = ctx->Rcart.as<double>();
  a.Rf32 = ctx->Rf32.as<double>();
  a.invdeg = ctx->invdeg.as<double>();
  a.isR0 = ctx->isR0.as<int>();
  a.nvec = ctx->nvec;
  a.w = w;
  a.kpt = ctx->kpt.as<double>();
  a.nk = ctx->nk;
  a.nv = ctx->nv;
  a.nc = ctx->nc;
  a.eig = ctx->eig.as<double>();
  a.U = ctx->U.as<double2>();
  a.eta32 = eta32;
  a.inv_sqrt2_f32 = (double)(1.0f / sqrtf(2.0f));
  a.h = ctx->h.as<double2>();
  a.N = ctx->N;
  const size_t need = (size_t)ctx->nvec * 16 + 3 * (size_t)w * w * 16 + (size_t)nb * w * 16 +
                      3 * (size_t)ctx->nv * w * 16;
  size_t smem = 0;
  int grid = 0;
  if (int r = place_work(ctx, need, ctx->nk, &a.gwork, &a.gstride, &smem, &grid)) return r;
  CK(cudaFuncSetAttribute(k_velocity, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_velocity<<<grid, kBandsThreads, smem, ctx->stream>>>(a); WTBG_COUNT(ctx, 1);
  CKL("k_velocity");
  return 0;
}

int launch_sp_table(wtbg_ctx* ctx, float* d_out) {
  const long long N = ctx->N;
  // scratch: rows (N*15 f32), key_in, key_out (N f32), idx_in, idx_out (N int), cub temp
  size_t cub_bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, (const float*)nullptr, (float*)nullptr,
                                  (const int*)nullptr, (int*)nullptr, (int)N);
  const size_t rows_b = (size_t)N * 15 * 4, vec_b = (size_t)N * 4;
  const size_t total = rows_b + 4 * vec_b + cub_bytes + 1024;
  ENSURE(ctx->tmp, total);
  char* base = ctx->tmp.as<char>();
  float* rows = reinterpret_cast<float*>(base);
  float* kin = reinterpret_cast<float*>(base + rows_b);
  float* kout = kin + N;
  int* iin = reinterpret_cast<int*>(kout + N);
  int* iout = iin + N;
  void* ctmp = reinterpret_cast<void*>(((uintptr_t)(iout + N) + 255) & ~(uintptr_t)255);
  const int th = 256;
  const int gr = (int)((N + th - 1) / th);
  const double* fd = nullptr;
  if (ctx->temp_on) {
    if (int r = ensure_fdeh(ctx, false)) return r;
    fd = ctx->fdeh.as<double>();
  }
  k_sp_rows<<<gr, th, 0, ctx->stream>>>(ctx->kpt.as<double>(), ctx->eig.as<double>(), ctx->nocp.as<int>(),
                                         ctx->h.as<double2>(), fd, ctx->nk, ctx->nv, ctx->nc, N, rows, kin, iin); WTBG_COUNT(ctx, 1);
  CKL("k_sp_rows");
  // LSD radix sort is stable: equal keys keep their original (quantumnumbers2) order,
  // which is what the strict-greater bubble sort produces.
  CK(cub::DeviceRadixSort::SortPairs(ctmp, cub_bytes, kin, kout, iin, iout, (int)N, 0, 32, ctx->stream));
  k_sp_gather<<<gr, th, 0, ctx->stream>>>(rows, iout, N, d_out); WTBG_COUNT(ctx, 1);
  CKL("k_sp_gather");
  return 0;
}

// Berry curvature of every k (berrycurv / berrycurvbz): eigsys of all bands, then k_berry
int launch_berry(wtbg_ctx* ctx, int nk, const double* d_kpt, const double* d_eig, const double2* d_U, const int* d_nocp,
                 double gamma, double degtol, double* d_out) {
  const int w = ctx->w, nvec = ctx->nvec;
  BerryArgs a;
  a.HR = ctx->HR.as<double2>();
  a.Rcart = ctx->Rcart.as<double>();
  a.Rf32 = ctx->Rf32.as<double>();
  a.invdeg = ctx->invdeg.as<double>();
  a.isR0 = ctx->isR0.as<int>();
  a.nvec = nvec;
  a.w = w;
  a.nk = nk;
  a.kpt = d_kpt;
  a.eig = d_eig;
  a.U = d_U;
  a.nocp = d_nocp;
  a.gamma2 = gamma * gamma;
  a.degtol = degtol;
  a.out = d_out;
  size_t smem = 0;
  int grid = 0;
  if (int r = place_work(ctx, sizeof(double2) * ((size_t)nvec + 5 * (size_t)w * w), nk, &a.gwork, &a.gstride, &smem,
                         &grid))
    return r;
  CK(cudaFuncSetAttribute(k_berry, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_berry<<<grid, kBandsThreads, smem, ctx->stream>>>(a); WTBG_COUNT(ctx, 1);
  CKL("k_berry");
  return 0;
}

// single-particle optical activity of every k (spoptpolbz): eigsys of all bands, then k_optbz
int launch_optbz(wtbg_ctx* ctx, int nk, int nv, int nc, const double* d_kpt, const double* d_eig, const double2* d_U,
                 const int* d_nocp, double sme, double* d_out, int* d_kstat) {
  const int w = ctx->w, nvec = ctx->nvec;
  OptBzArgs a;
  a.HR = ctx->HR.as<double2>();
  a.Rcart = ctx->Rcart.as<double>();
  a.Rf32 = ctx->Rf32.as<double>();
  a.invdeg = ctx->invdeg.as<double>();
  a.isR0 = ctx->isR0.as<int>();
  a.nvec = nvec;
  a.w = w;
  a.nk = nk;
  a.nv = nv;
  a.nc = nc;
  a.kpt = d_kpt;
  a.eig = d_eig;
  a.U = d_U;
  a.nocp = d_nocp;
  a.sme32 = (double)(float)sme;
  a.norm32 = (double)(1.0f / sqrtf(2.0f));
  a.out = d_out;
  a.kstat = d_kstat;
  size_t smem = 0;
  int grid = 0;
  if (int r = place_work(ctx, sizeof(double2) * ((size_t)nvec + 4 * (size_t)w * w), nk, &a.gwork, &a.gstride, &smem,
                         &grid))
    return r;
  CK(cudaFuncSetAttribute(k_optbz, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_optbz<<<grid, kBandsThreads, smem, ctx->stream>>>(a); WTBG_COUNT(ctx, 1);
  CKL("k_optbz");
  return 0;
}
