// Temperature BSE (BSET=T, BSET_BND=T): the occupation factor of each basis state
//   f_i = f_v - f_c,  f(E) = 1 / (exp(E / (kB T)) + 1),  E_F = 0
// (fermidisteh, subroutines/general_subs.f90:607-635), which scales the interaction part of
// every kernel row (matrizelbsetemp, bse_subs_temp.f90:2-126; matrizelbsekqtemp :128-337),
// the single-particle strengths (bse_solver-tool-diel-temp.f90:416-423) and one factor of the
// oscillator strengths (dielbseptemp, bse_subs_temp.f90:340-395).
#include "common.cuh"

namespace {

// kB as the reference's single-precision literal 8.617330350E-5
constexpr double kKB = (double)8.617330350e-5f;

__global__ void k_fdeh(const double* eigc, const double* eigv, int nk, int nv, int nc, double temp, double* f) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int ncv = nc * nv, nb = nc + nv;
  if (i >= (long long)nk * ncv) return;
  const long long k = i / ncv;
  const int c = (int)((i % ncv) / nv), v = (int)(i % nv);
  const double ec = eigc[k * nb + nv + c], ev = eigv[k * nb + v];
  const double beta = 1.0 / (kKB * temp);
  const double fv = 1.0 / (exp(ev * beta) + 1.0);
  const double fc = 1.0 / (exp(ec * beta) + 1.0);
  f[i] = fv - fc;
}

// g = [h (5 vectors) ; h * f (5 vectors)]
__global__ void k_g_temperature(const double2* h, const double* f, long long N, double2* g) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double fi = f[i];
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    const double2 x = h[a * N + i];
    g[a * N + i] = x;
    g[(5 + a) * N + i] = make_double2(x.x * fi, x.y * fi);
  }
}

}  // namespace

int ensure_fdeh(wtbg_ctx* ctx, bool q_mesh) {
  if (!ctx->temp_on) return WTBG_OK;
  const long long N = ctx->N;
  ENSURE(ctx->fdeh, (size_t)N * 8);
  // fermidisteh replaces T = 0 by the single-precision literal 1E-8
  const double t = (ctx->temp == 0.0) ? (double)1e-8f : ctx->temp;
  const double* eigc = q_mesh ? ctx->eigq.as<double>() : ctx->eig.as<double>();
  k_fdeh<<<(unsigned)((N + 255) / 256), 256, 0, ctx->stream>>>(eigc, ctx->eig.as<double>(), ctx->nk, ctx->nv, ctx->nc,
                                                               t, ctx->fdeh.as<double>());
  WTBG_COUNT(ctx, 1);
  CKL("k_fdeh");
  return WTBG_OK;
}

// With temperature the tridiagonal reduction carries ten vectors (g <- Q^T g): the five
// velocity vectors and the five f-weighted ones.
int fill_g_vectors(wtbg_ctx* ctx, double2* g) {
  const long long N = ctx->N;
  if (int r = ensure_fdeh(ctx, false)) return r;
  k_g_temperature<<<(unsigned)((N + 255) / 256), 256, 0, ctx->stream>>>(ctx->h.as<double2>(), ctx->fdeh.as<double>(),
                                                                        N, g);
  WTBG_COUNT(ctx, 1);
  CKL("k_g_temperature");
  return WTBG_OK;
}
