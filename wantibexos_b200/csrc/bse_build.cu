// Kernel (b): the exciton (BSE) kernel build.
//
// Reference: matrizelbse (subroutines/bse_subs.f90:2-124) called for every j >= i
// (subprograms/bse_solver-tool-diel.f90:431-458), and matrizelbsekq
// (subroutines/bse_subs_kpath.f90:1-208) for a centre-of-mass momentum Q.
// Element (i, j) with i = (k, c, v), j = (k', c', v') in quantumnumbers2 order:
//     H_ij = W(k - k') <c_i|c_j> <v_i|v_j>            (i != j; <a|b> = sum_m conj(a_m) b_m)
//     H_ii = (E_c - E_v) + W(0)
//   and for Q != 0 additionally  - W(Q) <c_i^{k+Q}|v_i> <v_j|c_j^{k'+Q}>  (exchange).
// The same expression gives both triangles of the Hermitian matrix, so the device stores
// the LOWER triangle (column-major, ld = N) that the tridiagonalisation reads.
//
// B200 design: one CTA per (k-block, k'-block) tile of the lower triangle.  The overlaps
// <c|c'> and <v|v'> of the tile are small complex GEMMs (K = w) computed once per tile in
// shared memory; the Coulomb factor W(k-k') is evaluated once per (k, k') pair; the
// Kronecker expansion into the (nc*nv) x (nc*nv) blocks happens in the store loop, so every
// element of the 16*N^2-byte matrix is written to HBM exactly once.  Off-diagonal tiles are
// staged in shared memory in chunks of CW columns (double-buffered, in the space the band
// vectors occupied) and leave through one TMA bulk tensor store per chunk, which overlaps the
// write of one chunk with the evaluation of the next; the TMA unit clips the rows past N of the
// last block row.  Diagonal tiles (lower half only) use plain coalesced 16-byte stores.  The
// kernel is bound by the HBM write of the matrix.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include <cudaTypedefs.h>

#include "common.cuh"
#include "coulomb.cuh"

namespace {

constexpr int kBuildThreads = 256;

struct BuildArgs {
  const double2* Uc;    // conduction eigenvectors [nk][nb][w] (k+Q mesh for Q != 0)
  const double2* Uv;    // valence eigenvectors   [nk][nb][w]
  const double* eigc;   // [nk][nb]
  const double* eigv;   // [nk][nb]
  const double* kpt;    // [nk][3]
  int nk, nv, nc, w, nb;
  CoulombDev P;
  int exch;
  double vq;
  const double2* vcv;   // [N] <c^{k+Q}|v> per state (exchange only)
  const double* fdeh;   // [N] occupation factor f_v - f_c (temperature BSE) or nullptr
  double2* H;
  long long N;
  int TK, nbk;
  // precision form: band overlaps from the tensor-core GEMM, FP32 [2n][n] (Re rows, then Im),
  // n = nk * nc (conduction) and nk * nv (valence); nullptr for the FP64 form
  const float* Oc;
  const float* Ov;
  // TMA-staged stores of the off-diagonal tiles: CW columns per chunk (0: plain stores only)
  int cw;
};

__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, const void* src, int x, int y) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"((unsigned)__cvta_generic_to_shared(src)), "r"(x), "r"(y)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
template <int N_>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N_) : "memory");
}

__global__ void __launch_bounds__(kBuildThreads) k_bse_build(const __grid_constant__ CUtensorMap tmH, BuildArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  const long long t = blockIdx.x;
  int bi = (int)floor((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((long long)(bi + 1) * (bi + 2) / 2 <= t) ++bi;
  while ((long long)bi * (bi + 1) / 2 > t) --bi;
  const int bj = (int)(t - (long long)bi * (bi + 1) / 2);
  const int TK = a.TK, nc = a.nc, nv = a.nv, w = a.w, nb = a.nb, ncv = nc * nv;
  const int kr0 = bi * TK, kc0 = bj * TK;
  const int nkr = min(TK, a.nk - kr0), nkc = min(TK, a.nk - kc0);
  const int tid = threadIdx.x, bs = blockDim.x;
  const int RC = TK * nc, RV = TK * nv;
  const int ws = w | 1;   // odd row stride: conflict-free 16-byte shared loads across rows

  // region 0: the band-vector rows, later the two store-staging buffers [CW][TK*ncv]
  double2* UcR = reinterpret_cast<double2*>(smem);
  double2* UcC = UcR + RC * ws;
  double2* UvR = UcC + RC * ws;
  double2* UvC = UvR + RV * ws;
  const int r0len = max(2 * RC * ws + 2 * RV * ws, 2 * ((a.cw * TK * ncv + 7) & ~7));
  double2* Mc = UcR + ((r0len + 7) & ~7);   // col-major [RC x RC], 128-byte aligned
  double2* Mv = Mc + RC * RC;          // col-major [RV x RV]
  double* Vt = reinterpret_cast<double*>(Mv + RV * RV);   // [kc][kr]
  double* dE = Vt + TK * TK;           // [TK*ncv]
  int* colinfo = reinterpret_cast<int*>(dE + TK * ncv);  // packed (kc, c', v') per tile column

  for (int it = a.Oc ? RC * w : tid; it < RC * w; it += bs) {
    const int kk = it / (nc * w), rem = it % (nc * w), c = rem / w, m = rem % w;
    const int row = kk * nc + c;
    UcR[row * ws + m] = (kk < nkr) ? a.Uc[((size_t)(kr0 + kk) * nb + nv + c) * w + m] : make_double2(0, 0);
    UcC[row * ws + m] = (kk < nkc) ? a.Uc[((size_t)(kc0 + kk) * nb + nv + c) * w + m] : make_double2(0, 0);
  }
  for (int it = a.Ov ? RV * w : tid; it < RV * w; it += bs) {
    const int kk = it / (nv * w), rem = it % (nv * w), v = rem / w, m = rem % w;
    const int row = kk * nv + v;
    UvR[row * ws + m] = (kk < nkr) ? a.Uv[((size_t)(kr0 + kk) * nb + v) * w + m] : make_double2(0, 0);
    UvC[row * ws + m] = (kk < nkc) ? a.Uv[((size_t)(kc0 + kk) * nb + v) * w + m] : make_double2(0, 0);
  }
  for (int it = tid; it < TK * TK; it += bs) {
    const int kc = it / TK, kr = it % TK;
    double v = 0.0;
    if (kr < nkr && kc < nkc) {
      const double* k1 = a.kpt + 3 * (size_t)(kr0 + kr);
      const double* k2 = a.kpt + 3 * (size_t)(kc0 + kc);
      v = coulomb_eval(a.P, k1[0] - k2[0], k1[1] - k2[1], k1[2] - k2[2]);
    }
    Vt[it] = v;
  }
  for (int it = tid; it < TK * ncv; it += bs) {
    const int kr = it / ncv, c = (it % ncv) / nv, v = it % nv;
    dE[it] = (kr < nkr) ? a.eigc[(size_t)(kr0 + kr) * nb + nv + c] - a.eigv[(size_t)(kr0 + kr) * nb + v] : 0.0;
    colinfo[it] = (kr << 16) | (c << 8) | v;
  }
  __syncthreads();
  if (a.Oc) {
    // precision form: the overlaps of this tile from the FP32 GEMM results
    const long long nC = (long long)a.nk * nc, nV = (long long)a.nk * nv;
    for (int it = tid; it < RC * RC; it += bs) {
      const int col = it / RC, row = it % RC;
      const int kr = row / nc, kc = col / nc;
      const long long i = (long long)kr0 * nc + row, j = (long long)kc0 * nc + col;
      Mc[it] = (kr < nkr && kc < nkc) ? make_double2((double)a.Oc[j * nC + i], (double)a.Oc[(nC + j) * nC + i])
                                      : make_double2(0, 0);
    }
    for (int it = tid; it < RV * RV; it += bs) {
      const int col = it / RV, row = it % RV;
      const int kr = row / nv, kc = col / nv;
      const long long i = (long long)kr0 * nv + row, j = (long long)kc0 * nv + col;
      Mv[it] = (kr < nkr && kc < nkc) ? make_double2((double)a.Ov[j * nV + i], (double)a.Ov[(nV + j) * nV + i])
                                      : make_double2(0, 0);
    }
  } else {
    for (int it = tid; it < RC * RC; it += bs) {
      const int col = it / RC, row = it % RC;
      const double2* x = UcR + row * ws;
      const double2* y = UcC + col * ws;
      double2 acc = make_double2(0, 0);
      for (int m = 0; m < w; ++m) acc = cadd(acc, cmulc(x[m], y[m]));
      Mc[it] = acc;
    }
    for (int it = tid; it < RV * RV; it += bs) {
      const int col = it / RV, row = it % RV;
      const double2* x = UvR + row * ws;
      const double2* y = UvC + col * ws;
      double2 acc = make_double2(0, 0);
      for (int m = 0; m < w; ++m) acc = cadd(acc, cmulc(x[m], y[m]));
      Mv[it] = acc;
    }
  }
  __syncthreads();

  const long long N = a.N;
  const long long I0 = (long long)kr0 * ncv, J0 = (long long)kc0 * ncv;
  const bool diag_tile = (bi == bj);
  const bool staged = a.cw > 0 && !diag_tile;
  // staged tiles evaluate all TK*ncv rows (those past N are clipped by the TMA store)
  const int rows = staged ? TK * ncv : nkr * ncv, cols = nkc * ncv;
  const int njp = bs / rows;
  const int ii = tid % rows;
  const bool thr_on = tid < njp * rows;
  const int kr = ii / ncv, c = (ii % ncv) / nv, v = ii % nv;
  const long long I = I0 + ii;
  const double2 vcvI = (a.exch && thr_on && I < N) ? a.vcv[I] : make_double2(0, 0);
  const double dEi = dE[ii];
  const double2* Mc_r = Mc + kr * nc + c;   // + col*RC
  const double2* Mv_r = Mv + kr * nv + v;   // + col*RV
  // element (I, J) of tile column jj
  auto elem = [&](int jj, long long J) -> double2 {
    const int ci = colinfo[jj];
    const int kc = ci >> 16, cc = (ci >> 8) & 0xff, vv = ci & 0xff;
    const double vk = Vt[kc * TK + kr];
    double2 val;
    if (a.fdeh == nullptr) {
      if (I == J) {
        val = make_double2(dEi + vk, 0.0);
      } else {
        val = cmul(cscale(Mc_r[(kc * nc + cc) * RC], vk), Mv_r[(kc * nv + vv) * RV]);
      }
      if (a.exch) {
        // vvc_j = conj(<c_j|v_j>) exactly
        const double2 t2 = cmul(cscale(vcvI, a.vq), cconj(a.vcv[J]));
        val = csub(val, t2);
      }
    } else {
      // temperature: the interaction part of the reference's upper-triangle row J (the
      // smaller index) is scaled by f_J; the band-energy difference is not
      double2 inter = (I == J) ? make_double2(vk, 0.0)
                               : cmul(cscale(Mc_r[(kc * nc + cc) * RC], vk), Mv_r[(kc * nv + vv) * RV]);
      if (a.exch) inter = csub(inter, cmul(cscale(vcvI, a.vq), cconj(a.vcv[J])));
      val = cscale(inter, a.fdeh[J]);
      if (I == J) val.x += dEi;
    }
    return val;
  };
  if (staged) {
    // off-diagonal tile (a full block column: cols = TK*ncv, a multiple of CW): chunk ch of CW
    // columns goes to buffer ch&1 and leaves with one store issued by thread 0.  One CTA
    // barrier per chunk: thread 0 reaches it only after the store of chunk ch-1 has finished
    // reading its buffer, which chunk ch+1 refills after that barrier; the store of chunk ch
    // proceeds while chunk ch+1 is evaluated into the other buffer.
    const int CW = a.cw;
    double2* stg = reinterpret_cast<double2*>(smem);
    const int bstride = (CW * rows + 7) & ~7;   // 128-byte aligned buffers
    for (int ch = 0; ch * CW < cols; ++ch) {
      double2* buf = stg + (size_t)(ch & 1) * bstride;
      if (thr_on)
        for (int cl = tid / rows; cl < CW; cl += njp) {
          const int jj = ch * CW + cl;
          buf[cl * rows + ii] = (I < N) ? elem(jj, J0 + jj) : make_double2(0, 0);
        }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      if (tid == 0) bulk_wait_read<0>();
      __syncthreads();
      if (tid == 0) tma_store_2d(&tmH, buf, (int)(2 * I0), (int)(J0 + (long long)ch * CW));
    }
    if (tid == 0) bulk_wait_read<0>();
    return;
  }
  if (!thr_on) return;
  double2* Hcol = a.H + I;
  for (int jj = tid / rows; jj < cols; jj += njp) {
    const long long J = J0 + jj;
    if (diag_tile && I < J) continue;
    Hcol[J * N] = elem(jj, J);
  }
}

__global__ void k_exchange_overlap(const double2* Uq, const double2* U, int nk, int nv, int nc, int w,
                                   double2* vcv) {
  const long long N = (long long)nk * nc * nv;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int nb = nc + nv, ncv = nc * nv;
  const int k = (int)(i / ncv), c = (int)((i % ncv) / nv), v = (int)(i % nv);
  const double2* x = Uq + ((size_t)k * nb + nv + c) * w;
  const double2* y = U + ((size_t)k * nb + v) * w;
  double2 acc = make_double2(0, 0);
  for (int m = 0; m < w; ++m) acc = cadd(acc, cmulc(x[m], y[m]));
  vcv[i] = acc;
}

// Columns per staged store chunk: the largest divisor of the tile width TK*ncv up to 16 whose
// two buffers fit in region 0 as sized by the band-vector rows (8 when region 0 must grow);
// 0 when a tile is taller than one TMA box (256 doubles) or wider than a 32-bit coordinate.
int build_cw(int TK, int nc, int nv, int w) {
  const int RC = TK * nc, RV = TK * nv, ncv = nc * nv, ws = w | 1, TR = TK * ncv;
  if (TR > 128) return 0;
  const long long u = 2LL * RC * ws + 2LL * RV * ws;
  int best = 0;
  for (int cw = 1; cw <= 16; ++cw)
    if (TR % cw == 0 && 2LL * ((cw * TR + 7) & ~7) <= u) best = cw;
  if (best >= 4) return best;
  for (int cw = 8; cw >= 1; --cw)
    if (TR % cw == 0) return cw;
  return 1;
}

size_t build_smem(int TK, int nc, int nv, int w) {
  const int RC = TK * nc, RV = TK * nv, ncv = nc * nv, ws = w | 1;
  const long long r0len = std::max(2LL * RC * ws + 2LL * RV * ws, 2LL * ((build_cw(TK, nc, nv, w) * TK * ncv + 7) & ~7));
  return 16ull * ((size_t)((r0len + 7) & ~7LL) + (size_t)RC * RC + (size_t)RV * RV) + 8ull * TK * TK +
         8ull * TK * ncv + 4ull * TK * ncv + 64;
}

}  // namespace

namespace {
PFN_cuTensorMapEncodeTiled_v12000 build_encode_fn() {
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

// H (N x N complex, column-major) as a FLOAT64 tensor {2N, N}; box = rows x cw of one staged chunk
int encode_h_map(wtbg_ctx* ctx, CUtensorMap* map, void* H, long long N, int rows, int cw) {
  auto fn = build_encode_fn();
  if (!fn) return set_err(ctx, WTBG_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  cuuint64_t dims[2] = {(cuuint64_t)(2 * N), (cuuint64_t)N};
  cuuint64_t strides[1] = {(cuuint64_t)(16 * N)};
  cuuint32_t box[2] = {(cuuint32_t)(2 * rows), (cuuint32_t)cw};
  cuuint32_t es[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, H, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return set_err(ctx, WTBG_ERR_CUDA, "bse_build: cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return WTBG_OK;
}
}  // namespace

CoulombDev make_coulomb_dev(const wtbg_coulomb* p, const double* L) {
  CoulombDev P{};
  P.type = p->coultype;
  P.ktol = p->ktol;
  const double a1[3] = {L[0], L[1], L[2]}, a2[3] = {L[3], L[4], L[5]}, a3[3] = {L[6], L[7], L[8]};
  const double vx[3] = {a1[1] * a2[2] - a1[2] * a2[1], a1[2] * a2[0] - a1[0] * a2[2],
                        a1[0] * a2[1] - a1[1] * a2[0]};
  const double vc2 = sqrt((vx[0] * vx[0]) + (vx[1] * vx[1]) + (vx[2] * vx[2]));
  const double vc3 = fabs(vx[0] * a3[0] + vx[1] * a3[1] + vx[2] * a3[2]);
  const int nkt = p->ngrid[0] * p->ngrid[1] * p->ngrid[2];
  P.vbz2d = 1.0 / (nkt * vc2);
  P.vbz3d = 1.0 / (nkt * vc3);
  const float cic32 = -(0.0904756f) * 1000.0f;
  P.cic = (double)cic32;
  const double pi32 = (double)acosf(-1.0f);
  // V2DRK (coulomb_pot.f90:311-319)
  const double epar = p->ediel[1], et = p->ediel[0], eb = p->ediel[2];
  P.eta = sqrt(epar / p->ez);
  P.kappa = sqrt(epar * p->ez);
  P.pb = (eb - P.kappa) / (eb + P.kappa);
  P.pt = (et - P.kappa) / (et + P.kappa);
  P.lc = p->lc;
  P.w = p->w;
  P.r0 = p->r0;
  P.ez = p->ez;
  // V2DK (coulomb_pot.f90:25-42)
  const double n1 = sqrt(a1[0] * a1[0] + a1[1] * a1[1] + a1[2] * a1[2]);
  const double n2 = sqrt(a2[0] * a2[0] + a2[1] * a2[1] + a2[2] * a2[2]);
  const double n3 = sqrt(a3[0] * a3[0] + a3[1] * a3[1] + a3[2] * a3[2]);
  const double a0 = 0.5 * (n1 + n2);
  P.v2dk_r0 = ((p->ediel[1] - 1.0) * p->lc) / (p->ediel[0] + p->ediel[2]);
  const double g1 = (double)(p->ngrid[0] * p->ngrid[1]);
  const double auxi = (2. * pi32 * P.v2dk_r0) / (a0 * sqrt(g1));
  P.v2dk_ed = (p->ediel[0] + p->ediel[2]) / (2.0);
  const double alpha1 = (double)1.76f, alpha2 = 1.0, alpha3 = 0.0;
  P.v2dk_q0 = P.vbz2d * (P.cic / P.v2dk_ed) * (a0 * sqrt(g1) / (2. * pi32)) *
              (alpha1 + auxi * alpha2 + alpha3 * auxi * auxi);
  // V3D / V3DL
  P.ed3 = (p->coultype == WTBG_V3DL) ? p->ediel[1] : 1.0;
  // V2DT
  P.rc = 0.5 * a3[2];
  // V0DT
  double cr = n1 < n2 ? n1 : n2;
  cr = cr < n3 ? cr : n3;
  P.cr = 0.5 * cr;
  // V1DT q -> 0 value (coulomb_pot.f90:414)
  P.v1dt_q0 = (P.vbz3d * P.cic) * ((p->lc * p->lc) / 16.0) * (2.0 * log(p->lc) - 1.0);
  return P;
}

// Precision form of the band overlaps <a_i|a_j> = sum_m conj(u_im) u_jm over all (k, band)
// rows of one band block as one real GEMM: A rows [Re u | Im u], B rows (Re out) [Re u | Im u]
// and (Im out) [Im u | -Re u], 3-term split-BF16 (segments padded to S, a multiple of 8).
__global__ void k_ovl_ops(const double2* U, int nk, int nb, int off, int cnt, int w, int S, __nv_bfloat16* A3,
                          __nv_bfloat16* B3) {
  const long long n = (long long)nk * cnt, i = blockIdx.x;
  const int k = (int)(i / cnt), b = (int)(i % cnt);
  __nv_bfloat16* ra = A3 + i * 6 * S;
  __nv_bfloat16* rr = B3 + i * 6 * S;
  __nv_bfloat16* ri = B3 + (n + i) * 6 * S;
  for (int m = threadIdx.x; m < S; m += blockDim.x) {
    const double2 u = (m < w) ? U[((size_t)k * nb + off + b) * w + m] : make_double2(0, 0);
    put_split_row(ra, 2 * S, m, u.x, true);
    put_split_row(ra, 2 * S, S + m, u.y, true);
    put_split_row(rr, 2 * S, m, u.x, false);
    put_split_row(rr, 2 * S, S + m, u.y, false);
    put_split_row(ri, 2 * S, m, u.y, false);
    put_split_row(ri, 2 * S, S + m, -u.x, false);
  }
}

// overlaps of the band block [off, off + cnt) of U on the tensor cores into out ([2n][n] FP32)
static int run_precision_overlaps(wtbg_ctx* ctx, const double2* U, int off, int cnt, DevBuf& out) {
  const int nk = ctx->nk, nb = ctx->nv + ctx->nc, w = ctx->w;
  const long long n = (long long)nk * cnt;
  const int S = (w + 7) / 8 * 8, K = 6 * S;
  if (n > 0x7fffffffLL / 2) return set_err(ctx, WTBG_ERR_UNSUPPORTED, "precision form: overlap GEMM too large");
  ENSURE(ctx->pOpA, (size_t)n * K * 2);
  ENSURE(ctx->pOpB, (size_t)2 * n * K * 2);
  ENSURE(out, (size_t)2 * n * n * 4);
  ENSURE(ctx->pErr, 16);
  k_ovl_ops<<<(unsigned)n, 64, 0, ctx->stream>>>(U, nk, nb, off, cnt, w, S, ctx->pOpA.as<__nv_bfloat16>(),
                                                 ctx->pOpB.as<__nv_bfloat16>());
  WTBG_COUNT(ctx, 1);
  CKL("k_ovl_ops");
  return gemm_bf16(ctx, ctx->pErr.as<int>(), ctx->pOpA.as<__nv_bfloat16>(), K, (int)n, K,
                   ctx->pOpB.as<__nv_bfloat16>(), K, (int)(2 * n), out.as<float>(), n, true);
}

// Builds the BSE matrix for Q = 0 (q4 == nullptr) or for a centre-of-mass momentum q4.
int launch_bse_build(wtbg_ctx* ctx, const wtbg_coulomb* p, const double* q4) {
  const int nc = ctx->nc, nv = ctx->nv, w = ctx->w, ncv = nc * nv;
  if (ncv > 256) return set_err(ctx, WTBG_ERR_UNSUPPORTED, "bse_build: nc*nv > 256");
  int TK = 128 / ncv;
  if (TK < 1) TK = 1;
  while (TK > 1 && build_smem(TK, nc, nv, w) > 96 * 1024) --TK;
  const size_t smem = build_smem(TK, nc, nv, w);
  if (smem > 200 * 1024) return set_err(ctx, WTBG_ERR_UNSUPPORTED, "bse_build: tile does not fit in shared memory");
  BuildArgs a;
  const bool q = (q4 != nullptr);
  a.Uc = q ? ctx->Uq.as<double2>() : ctx->U.as<double2>();
  a.Uv = ctx->U.as<double2>();
  a.eigc = q ? ctx->eigq.as<double>() : ctx->eig.as<double>();
  a.eigv = ctx->eig.as<double>();
  a.kpt = ctx->kpt.as<double>();
  a.nk = ctx->nk;
  a.nv = nv;
  a.nc = nc;
  a.w = w;
  a.nb = nc + nv;
  a.P = make_coulomb_dev(p, ctx->rlat);
  a.exch = 0;
  a.vq = 0.0;
  a.fdeh = nullptr;
  if (ctx->temp_on) {
    if (int r = ensure_fdeh(ctx, q)) return r;
    a.fdeh = ctx->fdeh.as<double>();
  }
  a.vcv = nullptr;
  a.Oc = a.Ov = nullptr;
  if (ctx->prec == 1) {
    if (int r = run_precision_overlaps(ctx, a.Uc, nv, nc, ctx->pOc)) return r;
    if (int r = run_precision_overlaps(ctx, a.Uv, 0, nv, ctx->pOv)) return r;
    a.Oc = ctx->pOc.as<float>();
    a.Ov = ctx->pOv.as<float>();
  }
  a.H = ctx->H.as<double2>();
  a.N = ctx->N;
  a.TK = TK;
  a.nbk = (ctx->nk + TK - 1) / TK;
  // TMA-staged stores for the off-diagonal tiles (there are none with a single block row)
  CUtensorMap tmH;
  memset(&tmH, 0, sizeof(tmH));
  a.cw = (a.nbk > 1 && 2 * a.N < 0x7fffffffLL) ? build_cw(TK, nc, nv, w) : 0;
  if (a.cw > 0)
    if (int r = encode_h_map(ctx, &tmH, a.H, a.N, TK * ncv, a.cw)) return r;
  if (q) {
    const double modq = sqrt((q4[1]) * (q4[1]) + (q4[2]) * (q4[2]) + (q4[3]) * (q4[3]));
    if (modq != 0.0) {
      // W(Q) = coulomb(vq, 0) on the host (single value, same formulas)
      ENSURE(ctx->tmp2, (size_t)ctx->N * 16 + 64);
      a.vcv = ctx->tmp2.as<double2>();
      const int th = 256;
      k_exchange_overlap<<<(int)((ctx->N + th - 1) / th), th, 0, ctx->stream>>>(
          ctx->Uq.as<double2>(), ctx->U.as<double2>(), ctx->nk, nv, nc, w, ctx->tmp2.as<double2>()); WTBG_COUNT(ctx, 1);
      CKL("k_exchange_overlap");
      a.exch = 1;
    }
  }
  if (a.exch) {
    // evaluate W(Q) with the device formula for exact agreement with the in-kernel values
    extern int eval_coulomb_single(wtbg_ctx*, const CoulombDev&, double, double, double, double*);
    double vq = 0.0;
    int r = eval_coulomb_single(ctx, a.P, q4[1], q4[2], q4[3], &vq);
    if (r) return r;
    a.vq = vq;
  }
  CK(cudaFuncSetAttribute(k_bse_build, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long ntile = (long long)a.nbk * (a.nbk + 1) / 2;
  if (ntile > 0x7fffffffLL) return set_err(ctx, WTBG_ERR_UNSUPPORTED, "bse_build: too many tiles");
  const bool prof = ctx->profiling != 0;
  if (prof) {
    if (int r = ensure_events(ctx, 2)) return r;
    cudaEventRecord(ctx->evpool[0], ctx->stream);
  }
  k_bse_build<<<(unsigned)ntile, kBuildThreads, smem, ctx->stream>>>(tmH, a); WTBG_COUNT(ctx, 1);
  CKL("k_bse_build");
  if (prof) {
    cudaEventRecord(ctx->evpool[1], ctx->stream);
    CK(cudaEventSynchronize(ctx->evpool[1]));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, ctx->evpool[0], ctx->evpool[1]));
    ctx->stats.build_ms += t;
    ctx->stats.build_bytes += (double)ctx->N * ((double)ctx->N + 1.0) * 0.5 * 16.0;
    ctx->stats.build_launches += 1;
  }
  return 0;
}

namespace {
__global__ void k_coulomb_single(CoulombDev P, double x, double y, double z, double* out) {
  *out = coulomb_eval(P, x, y, z);
}
}  // namespace

int eval_coulomb_single(wtbg_ctx* ctx, const CoulombDev& P, double x, double y, double z, double* out) {
  ENSURE(ctx->istat, 64);
  double* d = ctx->istat.as<double>();
  k_coulomb_single<<<1, 1, 0, ctx->stream>>>(P, x, y, z, d); WTBG_COUNT(ctx, 1);
  CKL("k_coulomb_single");
  CK(cudaMemcpyAsync(out, d, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}
