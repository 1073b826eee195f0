// C-ABI of libwtbgpu.so: context management, argument checks, host <-> device transfers
// and the order of kernel launches for each replaced reference stage (see wtbgpu.h).
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

int set_err(wtbg_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

int cuda_fail(wtbg_ctx* c, cudaError_t e, const char* where) {
  std::string m = std::string(where) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return set_err(c, WTBG_ERR_OOM, m);
  return set_err(c, WTBG_ERR_CUDA, m);
}

int ensure(wtbg_ctx* c, DevBuf& b, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (b.bytes >= bytes) return 0;
  if (b.p) {
    cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
  }
  cudaError_t e = cudaMalloc(&b.p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    b.p = nullptr;
    char msg[160];
    snprintf(msg, sizeof msg, "device allocation of %zu bytes failed", bytes);
    return set_err(c, WTBG_ERR_OOM, msg);
  }
  b.bytes = bytes;
  return 0;
}

namespace {

void free_buf(DevBuf& b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
}

}  // namespace

int ensure_events(wtbg_ctx* ctx, size_t n) {
  while (ctx->evpool.size() < n) {
    cudaEvent_t e;
    cudaError_t r = cudaEventCreate(&e);
    if (r != cudaSuccess) return cuda_fail(ctx, r, "cudaEventCreate");
    ctx->evpool.push_back(e);
  }
  return 0;
}

// device flag of the precision-form GEMMs (a pipeline wait that timed out)
int check_gemm_err(wtbg_ctx* ctx) {
  if (!ctx->prec || !ctx->pErr.p) return 0;
  int e = 0;
  CK(cudaMemcpyAsync(&e, ctx->pErr.p, 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (e) {
    CK(cudaMemsetAsync(ctx->pErr.p, 0, 4, ctx->stream));
    return set_err(ctx, WTBG_ERR_CUDA, "precision form: a tensor-core pipeline wait timed out");
  }
  return 0;
}

extern "C" {

int wtbg_set_reduction(wtbg_ctx* ctx, int mode) {
  if (!ctx || mode < 0 || mode > 3) return WTBG_ERR_ARG;
  ctx->tri_mode = (mode == 3) ? 2 : mode;
  ctx->bulge_warp_mode = (mode == 3) ? 1 : 0;
  return WTBG_OK;
}

int wtbg_set_profiling(wtbg_ctx* ctx, int on) {
  if (!ctx) return WTBG_ERR_ARG;
  ctx->profiling = on ? 1 : 0;
  return WTBG_OK;
}

int wtbg_get_stats(const wtbg_ctx* ctx, wtbg_stats* out) {
  if (!ctx || !out) return WTBG_ERR_ARG;
  *out = ctx->stats;
  return WTBG_OK;
}

int wtbg_reset_stats(wtbg_ctx* ctx) {
  if (!ctx) return WTBG_ERR_ARG;
  ctx->stats = wtbg_stats{};
  return WTBG_OK;
}

const char* wtbg_error_string(int s) {
  switch (s) {
    case WTBG_OK: return "ok";
    case WTBG_ERR_ARG: return "invalid argument";
    case WTBG_ERR_CUDA: return "CUDA error";
    case WTBG_ERR_OOM: return "out of device memory";
    case WTBG_ERR_NOCONV: return "iterative solver did not converge";
    case WTBG_ERR_STATE: return "call order violated";
    case WTBG_ERR_BANDWINDOW: return "Number of valence/conduction states higher than occupied/unoccupied states";
    case WTBG_ERR_NOEMPTY: return "no eigenvalue above the Fermi level";
    case WTBG_ERR_UNSUPPORTED: return "unsupported size or option";
    case WTBG_ERR_NOCUDA: return "no CUDA device";
    default: return "unknown status";
  }
}

const char* wtbg_last_error(const wtbg_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

double wtbg_last_device_ms(const wtbg_ctx* ctx) { return ctx ? ctx->last_ms : 0.0; }

int wtbg_create(wtbg_ctx** out, int device) {
  if (!out) return WTBG_ERR_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return WTBG_ERR_NOCUDA;
  }
  if (device < 0 || device >= n) return WTBG_ERR_ARG;
  wtbg_ctx* ctx = new wtbg_ctx();
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess) {
    cudaGetLastError();
    delete ctx;
    return WTBG_ERR_CUDA;
  }
  *out = ctx;
  return WTBG_OK;
}

int wtbg_destroy(wtbg_ctx* ctx) {
  if (!ctx) return WTBG_ERR_ARG;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  DevBuf* bufs[] = {&ctx->HR, &ctx->Rcart, &ctx->Rf32, &ctx->invdeg, &ctx->isR0, &ctx->kpt, &ctx->eig, &ctx->U,
                    &ctx->nocp, &ctx->kstat, &ctx->kptq, &ctx->eigq, &ctx->Uq, &ctx->nocpq, &ctx->h, &ctx->H,
                    &ctx->d, &ctx->e, &ctx->tau, &ctx->g, &ctx->fdeh, &ctx->Wp, &ctx->slots, &ctx->part, &ctx->scal,
                    &ctx->yv, &ctx->lam, &ctx->bgrid, &ctx->ws, &ctx->act, &ctx->zsel, &ctx->csz, &ctx->sp_in, &ctx->sp_out,
                    &ctx->sp_om, &ctx->tmp, &ctx->tmp2, &ctx->istat, &ctx->pOpA, &ctx->pOpB,
                    &ctx->pHk, &ctx->pOc, &ctx->pOv, &ctx->pErr, &ctx->triErr, &ctx->gwork,
                    &ctx->t2V, &ctx->t2X, &ctx->t2D, &ctx->t2G, &ctx->t2T, &ctx->t2P, &ctx->t2AB, &ctx->t2prog, &ctx->t2de};
  for (DevBuf* b : bufs) free_buf(*b);
  for (cudaEvent_t e : ctx->evpool) cudaEventDestroy(e);
  if (ctx->tri_exec) cudaGraphExecDestroy(ctx->tri_exec);
  cudaEventDestroy(ctx->ev0);
  cudaEventDestroy(ctx->ev1);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return WTBG_OK;
}

int wtbg_set_model(wtbg_ctx* ctx, int w, int nvec, const double* hre, const double* him, const int* rvec,
                   const int* deg, const double* rlat, double efermi, double scs) {
  if (!ctx) return WTBG_ERR_ARG;
  if (w <= 0 || nvec <= 0 || !hre || !him || !rvec || !deg || !rlat)
    return set_err(ctx, WTBG_ERR_ARG, "set_model: bad sizes or null pointers");
  if (w > WTBG_MAX_W) return set_err(ctx, WTBG_ERR_UNSUPPORTED, "set_model: w exceeds the per-k eigensolver limit");
  for (int i = 0; i < nvec; ++i)
    if (deg[i] == 0) return set_err(ctx, WTBG_ERR_ARG, "set_model: zero degeneracy");
  if (int r = set_device(ctx)) return r;
  ctx->w = w;
  ctx->nvec = nvec;
  for (int i = 0; i < 3; ++i)
    for (int c = 0; c < 3; ++c) ctx->rlat[i * 3 + c] = rlat[i + 3 * c];   // Fortran rlat(i,c)
  ctx->efermi = efermi;
  ctx->scs = scs;
  const size_t ww = (size_t)w * w;
  std::vector<double2> hr(nvec * ww);
  std::vector<double> rc(3 * (size_t)nvec), rf(3 * (size_t)nvec), inv(nvec);
  std::vector<int> is0(nvec);
  for (int iR = 0; iR < nvec; ++iR) {
    for (int n = 0; n < w; ++n)
      for (int m = 0; m < w; ++m) {
        const size_t src = (size_t)iR + (size_t)nvec * ((size_t)m + (size_t)w * n);   // hopmatrices(iR,m,n)
        hr[iR * ww + (size_t)n * w + m] = make_double2(hre[src], him[src]);
      }
    const int r1 = rvec[iR], r2 = rvec[iR + nvec], r3 = rvec[iR + 2 * nvec];
    for (int c = 0; c < 3; ++c) {
      // (r1*a1c + r2*a2c) + r3*a3c, as the reference's expression is evaluated
      const double v = (r1 * ctx->rlat[0 * 3 + c] + r2 * ctx->rlat[1 * 3 + c]) + r3 * ctx->rlat[2 * 3 + c];
      rc[3 * iR + c] = v;
      rf[3 * iR + c] = (double)(float)v;
    }
    inv[iR] = 1.0 / (double)deg[iR];
    is0[iR] = (r1 == 0 && r2 == 0 && r3 == 0) ? 1 : 0;
  }
  ENSURE(ctx->HR, hr.size() * 16);
  ENSURE(ctx->Rcart, rc.size() * 8);
  ENSURE(ctx->Rf32, rf.size() * 8);
  ENSURE(ctx->invdeg, inv.size() * 8);
  ENSURE(ctx->isR0, is0.size() * 4);
  CK(cudaMemcpyAsync(ctx->HR.p, hr.data(), hr.size() * 16, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->Rcart.p, rc.data(), rc.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->Rf32.p, rf.data(), rf.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->invdeg.p, inv.data(), inv.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->isR0.p, is0.data(), is0.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->have_bands = ctx->have_velocity = ctx->have_matrix = ctx->have_solution = false;
  ctx->fast_ready = false;
  return WTBG_OK;
}

static int check_kstat(wtbg_ctx* ctx, int nk) {
  std::vector<int> st(nk);
  CK(cudaMemcpyAsync(st.data(), ctx->kstat.p, (size_t)nk * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  for (int k = 0; k < nk; ++k) {
    if (st[k] == 1) return set_err(ctx, WTBG_ERR_NOCONV, "bands: Jacobi sweep cap reached at k-point " + std::to_string(k + 1));
    if (st[k] == 2) return set_err(ctx, WTBG_ERR_NOEMPTY, "bands: no eigenvalue above E_F at k-point " + std::to_string(k + 1));
    if (st[k] == 3)
      return set_err(ctx, WTBG_ERR_BANDWINDOW, "bands: nv/nc exceed occupied/unoccupied states at k-point " + std::to_string(k + 1));
  }
  return 0;
}

int wtbg_bands(wtbg_ctx* ctx, int nk, const double* kpt, int nv, int nc, double* eigv, double* vector, int* nocpk,
               double* egap) {
  if (!ctx) return WTBG_ERR_ARG;
  if (ctx->w == 0) return set_err(ctx, WTBG_ERR_STATE, "bands: no model");
  if (nk <= 0 || nv <= 0 || nc <= 0 || !kpt) return set_err(ctx, WTBG_ERR_ARG, "bands: bad sizes");
  if (nv + nc > ctx->w) return set_err(ctx, WTBG_ERR_BANDWINDOW, "bands: nv + nc > w");
  if (int r = set_device(ctx)) return r;
  ctx->nk = nk;
  ctx->nv = nv;
  ctx->nc = nc;
  const int nb = nv + nc, w = ctx->w;
  ctx->N = (long long)nk * nc * nv;
  std::vector<double> kp(3 * (size_t)nk);
  for (int k = 0; k < nk; ++k)
    for (int c = 0; c < 3; ++c) kp[3 * k + c] = kpt[k + (size_t)nk * c];
  ENSURE(ctx->kpt, kp.size() * 8);
  ENSURE(ctx->eig, (size_t)nk * nb * 8);
  ENSURE(ctx->U, (size_t)nk * nb * w * 16);
  ENSURE(ctx->nocp, (size_t)nk * 4);
  ENSURE(ctx->kstat, (size_t)nk * 4);
  Timer t(ctx);
  CK(cudaMemcpyAsync(ctx->kpt.p, kp.data(), kp.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
  if (int r = launch_bands(ctx, false)) return r;
  if (int r = t.stop()) return r;
  if (int r = check_kstat(ctx, nk)) return r;
  if (int r = check_gemm_err(ctx)) return r;
  ctx->have_bands = true;
  ctx->have_velocity = ctx->have_matrix = ctx->have_solution = false;
  ctx->fast_ready = false;
  std::vector<double> e((size_t)nk * nb);
  CK(cudaMemcpyAsync(e.data(), ctx->eig.p, e.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
  std::vector<int> no(nk);
  CK(cudaMemcpyAsync(no.data(), ctx->nocp.p, (size_t)nk * 4, cudaMemcpyDeviceToHost, ctx->stream));
  std::vector<double2> u;
  if (vector) {
    u.resize((size_t)nk * nb * w);
    CK(cudaMemcpyAsync(u.data(), ctx->U.p, u.size() * 16, cudaMemcpyDeviceToHost, ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  double gap = 50.0;
  for (int k = 0; k < nk; ++k) {
    const double gk = e[(size_t)k * nb + nv] - e[(size_t)k * nb + nv - 1];
    if (gk <= gap) gap = gk;
  }
  if (egap) *egap = gap;
  if (eigv)
    for (int k = 0; k < nk; ++k)
      for (int j = 0; j < nb; ++j) eigv[k + (size_t)nk * j] = e[(size_t)k * nb + j];
  if (nocpk)
    for (int k = 0; k < nk; ++k) nocpk[k] = no[k];
  if (vector)
    for (int k = 0; k < nk; ++k)
      for (int j = 0; j < nb; ++j)
        for (int m = 0; m < w; ++m) {
          const double2 v = u[((size_t)k * nb + j) * w + m];
          const size_t dst = (size_t)k + (size_t)nk * ((size_t)j + (size_t)nb * m);   // vector(k, j, m)
          vector[2 * dst] = v.x;
          vector[2 * dst + 1] = v.y;
        }
  return WTBG_OK;
}

int wtbg_velocity(wtbg_ctx* ctx, double sme, double* hr) {
  if (!ctx) return WTBG_ERR_ARG;
  if (!ctx->have_bands) return set_err(ctx, WTBG_ERR_STATE, "velocity: call wtbg_bands first");
  if (int r = set_device(ctx)) return r;
  const long long N = ctx->N;
  ENSURE(ctx->h, (size_t)N * 5 * 16);
  Timer t(ctx);
  // cmplx(0.0, sme) without KIND: the broadening enters as float32 (optics.f90:139)
  if (int r = launch_velocity(ctx, (double)(float)sme)) return r;
  if (int r = t.stop()) return r;
  ctx->have_velocity = true;
  if (hr) CK(cudaMemcpy(hr, ctx->h.p, (size_t)N * 5 * 16, cudaMemcpyDeviceToHost));
  return WTBG_OK;
}

int wtbg_sp_table(wtbg_ctx* ctx, float* vecres) {
  if (!ctx || !vecres) return WTBG_ERR_ARG;
  if (!ctx->have_velocity) return set_err(ctx, WTBG_ERR_STATE, "sp_table: call wtbg_velocity first");
  if (int r = set_device(ctx)) return r;
  const long long N = ctx->N;
  ENSURE(ctx->sp_in, (size_t)N * 15 * 4);
  Timer t(ctx);
  if (int r = launch_sp_table(ctx, ctx->sp_in.as<float>())) return r;
  if (int r = t.stop()) return r;
  CK(cudaMemcpy(vecres, ctx->sp_in.p, (size_t)N * 15 * 4, cudaMemcpyDeviceToHost));
  return WTBG_OK;
}

int wtbg_bse_build(wtbg_ctx* ctx, const wtbg_coulomb* p) {
  if (!ctx || !p) return WTBG_ERR_ARG;
  if (!ctx->have_bands) return set_err(ctx, WTBG_ERR_STATE, "bse_build: call wtbg_bands first");
  if (p->coultype < WTBG_V2DK || p->coultype > WTBG_V0DT) return set_err(ctx, WTBG_ERR_ARG, "Wrong Coulomb Potential");
  if (int r = set_device(ctx)) return r;
  const long long N = ctx->N;
  ENSURE(ctx->H, (size_t)N * N * 16);
  Timer t(ctx);
  if (int r = launch_bse_build(ctx, p, nullptr)) return r;
  if (int r = t.stop()) return r;
  if (int r = check_gemm_err(ctx)) return r;
  ctx->have_matrix = true;
  ctx->fast_ready = false;
  ctx->have_solution = false;
  return WTBG_OK;
}

int wtbg_bse_get_matrix(wtbg_ctx* ctx, double* hbse) {
  if (!ctx || !hbse) return WTBG_ERR_ARG;
  if (!ctx->have_matrix || ctx->have_solution) return set_err(ctx, WTBG_ERR_STATE, "bse_get_matrix: no built matrix");
  if (int r = set_device(ctx)) return r;
  const long long N = ctx->N;
  std::vector<double2> L((size_t)N * N);
  CK(cudaMemcpy(L.data(), ctx->H.p, (size_t)N * N * 16, cudaMemcpyDeviceToHost));
  for (long long j = 0; j < N; ++j)
    for (long long i = 0; i < N; ++i) {
      double2 v = make_double2(0, 0);
      if (j >= i) {
        const double2 l = L[j + i * N];   // lower element (j, i)
        v = make_double2(l.x, -l.y);
      }
      hbse[2 * (i + j * N)] = v.x;
      hbse[2 * (i + j * N) + 1] = v.y;
    }
  return WTBG_OK;
}

int wtbg_bse_solve(wtbg_ctx* ctx, int dtfull, int cpol, double* W, double* act) {
  if (!ctx) return WTBG_ERR_ARG;
  if (!ctx->have_matrix) return set_err(ctx, WTBG_ERR_STATE, "bse_solve: call wtbg_bse_build first");
  if (!ctx->have_velocity && act) return set_err(ctx, WTBG_ERR_STATE, "bse_solve: call wtbg_velocity first");
  if (int r = set_device(ctx)) return r;
  const long long N = ctx->N;
  Timer t(ctx);
  if (int r = run_tridiagonalise(ctx)) return r;
  ctx->have_matrix = false;   // overwritten by the reflectors
  ctx->fast_ready = false;
  if (int r = run_tridiagonal_solve(ctx, dtfull, cpol, act != nullptr)) return r;
  if (int r = t.stop()) return r;
  ctx->have_solution = true;
  if (W) memcpy(W, ctx->lam_host.data(), (size_t)N * 8);
  if (act) CK(cudaMemcpy(act, ctx->act.p, (size_t)N * 8 * 8, cudaMemcpyDeviceToHost));
  return WTBG_OK;
}

int wtbg_bse_davidson(wtbg_ctx* ctx, int nev, int nb, int largest, int max_iter, double tol, const double* X0,
                      int dtfull, int cpol, double* W, double* act, double* X, int* iters, double* maxres) {
  if (!ctx || !W) return WTBG_ERR_ARG;
  if (!ctx->have_matrix) return set_err(ctx, WTBG_ERR_STATE, "bse_davidson: call wtbg_bse_build first");
  if (act && !ctx->have_velocity) return set_err(ctx, WTBG_ERR_STATE, "bse_davidson: call wtbg_velocity first");
  if (act && ctx->temp_on)
    return set_err(ctx, WTBG_ERR_UNSUPPORTED, "bse_davidson: oscillators with temperature come from wtbg_bse_solve");
  if (nev < 1 || nev > ctx->N || nb > ctx->N || max_iter < 1 || !(tol > 0))
    return set_err(ctx, WTBG_ERR_ARG, "bse_davidson: bad arguments");
  if (int r = set_device(ctx)) return r;
  const long long N = ctx->N;
  Timer t(ctx);
  double2* dX0 = nullptr;
  if (X0) {
    ENSURE(ctx->zsel, (size_t)N * nb * 16);
    dX0 = ctx->zsel.as<double2>();
    CK(cudaMemcpyAsync(dX0, X0, (size_t)N * nb * 16, cudaMemcpyHostToDevice, ctx->stream));
  }
  double2* dX = nullptr;
  if (X) {
    ENSURE(ctx->yv, (size_t)N * nev * 16);
    dX = ctx->yv.as<double2>();
  }
  std::vector<double> w, ac;
  int it = 0;
  double mr = 0.0;
  if (int r = run_davidson(ctx, nev, nb, largest, max_iter, tol, dX0, dtfull, cpol, w, ac, dX, &it, &mr)) return r;
  if (ctx->fast_mode)
    if (int r = fast_check(ctx)) return r;
  if (int r = t.stop()) return r;
  memcpy(W, w.data(), (size_t)nev * 8);
  if (act) memcpy(act, ac.data(), (size_t)nev * 8 * 8);
  if (X) CK(cudaMemcpy(X, dX, (size_t)N * nev * 16, cudaMemcpyDeviceToHost));
  if (iters) *iters = it;
  if (maxres) *maxres = mr;
  if (mr >= tol) return set_err(ctx, WTBG_ERR_NOCONV, "bse_davidson: residual above tolerance after max_iter");
  return WTBG_OK;
}

// gauge of an exciton vector for the BSE_WF files: unit norm, last component real and >= 0
// (the convention of wtbg_bse_eigvecs)
static void gauge_last_real(double* x, long long N) {
  double nrm = 0.0;
  for (long long i = 0; i < N; ++i) nrm += x[2 * i] * x[2 * i] + x[2 * i + 1] * x[2 * i + 1];
  const double lr = x[2 * (N - 1)], li = x[2 * (N - 1) + 1];
  const double r = std::hypot(lr, li);
  double cr = 1.0, ci = 0.0;   // multiply by conj(last)/|last|
  if (r > 0.0) {
    cr = lr / r;
    ci = -li / r;
  }
  const double s = nrm > 0.0 ? 1.0 / std::sqrt(nrm) : 1.0;
  for (long long i = 0; i < N; ++i) {
    const double a = x[2 * i], b = x[2 * i + 1];
    x[2 * i] = s * (a * cr - b * ci);
    x[2 * i + 1] = s * (a * ci + b * cr);
  }
  x[2 * (N - 1) + 1] = 0.0;
}

int wtbg_bse_lowest(wtbg_ctx* ctx, int nev, int nb, int max_iter, double tol, const double* X0, int dtfull, int cpol,
                    double* W, double* act, double* X, int* iters, double* maxres, int* used_dense) {
  if (!ctx || !W || !used_dense) return WTBG_ERR_ARG;
  *used_dense = 0;
  if (!ctx->have_matrix) return set_err(ctx, WTBG_ERR_STATE, "bse_lowest: call wtbg_bse_build first");
  const long long N = ctx->N;
  if (nev < 1 || nev > N) return set_err(ctx, WTBG_ERR_ARG, "bse_lowest: bad nev");
  int it = 0;
  double mr = 0.0;
  int st = WTBG_ERR_NOCONV;
  if (!ctx->temp_on || !act)
    st = wtbg_bse_davidson(ctx, nev, nb, 0, max_iter, tol, X0, dtfull, cpol, W, act, X, &it, &mr);
  if (iters) *iters = it;
  if (maxres) *maxres = mr;
  if (st == WTBG_OK) {
    if (X)
      for (int n = 0; n < nev; ++n) gauge_last_real(X + 2 * (size_t)N * n, N);
    return WTBG_OK;
  }
  if (st != WTBG_ERR_NOCONV && st != WTBG_ERR_UNSUPPORTED) return st;
  // dense FP64 fallback: every eigenpair of the same matrix, the nev lowest returned
  ctx->stats.dav_fallbacks += 1;
  *used_dense = 1;
  std::vector<double> w((size_t)N), a(act ? (size_t)N * 8 : 0);
  if (int r = wtbg_bse_solve(ctx, dtfull, cpol, w.data(), act ? a.data() : nullptr)) return r;
  const double ms = ctx->last_ms;
  memcpy(W, w.data(), (size_t)nev * 8);
  if (act)
    for (int c = 0; c < 8; ++c) memcpy(act + (size_t)nev * c, a.data() + (size_t)N * c, (size_t)nev * 8);
  if (X) {
    if (int r = wtbg_bse_eigvecs(ctx, 1, nev, X)) return r;
    ctx->last_ms += ms;
  }
  return WTBG_OK;
}

int wtbg_bands_batch(wtbg_ctx* const* ctxs, int nmod, const int* nk, const double* const* kpt, const int* nv,
                     const int* nc, double* egap) {
  if (!ctxs || nmod < 1 || !nk || !kpt || !nv || !nc) return WTBG_ERR_ARG;
  wtbg_ctx* ctx = ctxs[0];
  if (!ctx) return WTBG_ERR_ARG;
  for (int m = 0; m < nmod; ++m) {
    wtbg_ctx* c = ctxs[m];
    if (!c || c->device != ctx->device) return set_err(ctx, WTBG_ERR_ARG, "bands_batch: contexts must share a device");
    if (c->w == 0) return set_err(ctx, WTBG_ERR_STATE, "bands_batch: a context has no model");
    if (nk[m] <= 0 || nv[m] <= 0 || nc[m] <= 0 || !kpt[m] || nv[m] + nc[m] > c->w)
      return set_err(ctx, WTBG_ERR_ARG, "bands_batch: bad sizes for model " + std::to_string(m));
  }
  if (int r = set_device(ctx)) return r;
  Timer t(ctx);
  for (int m = 0; m < nmod; ++m) {
    wtbg_ctx* c = ctxs[m];
    c->nk = nk[m];
    c->nv = nv[m];
    c->nc = nc[m];
    c->N = (long long)nk[m] * nc[m] * nv[m];
    const int nb = nv[m] + nc[m];
    std::vector<double> kp(3 * (size_t)nk[m]);
    for (int k = 0; k < nk[m]; ++k)
      for (int a = 0; a < 3; ++a) kp[3 * k + a] = kpt[m][k + (size_t)nk[m] * a];
    if (int r = ensure(c, c->kpt, kp.size() * 8)) return r;
    if (int r = ensure(c, c->eig, (size_t)nk[m] * nb * 8)) return r;
    if (int r = ensure(c, c->U, (size_t)nk[m] * nb * c->w * 16)) return r;
    if (int r = ensure(c, c->nocp, (size_t)nk[m] * 4)) return r;
    if (int r = ensure(c, c->kstat, (size_t)nk[m] * 4)) return r;
    // every upload on the launching stream, so the batch kernel sees them in order
    CK(cudaMemcpyAsync(c->kpt.p, kp.data(), kp.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  if (int r = launch_bands_batch(ctxs, nmod)) return r;
  if (int r = t.stop()) return r;
  for (int m = 0; m < nmod; ++m) {
    wtbg_ctx* c = ctxs[m];
    if (int r = check_kstat(c, nk[m])) return set_err(ctx, r, "bands_batch: model " + std::to_string(m) + ": " + c->err);
    c->have_bands = true;
    c->have_velocity = c->have_matrix = c->have_solution = false;
    c->fast_ready = false;
    if (egap) {
      const int nb = nv[m] + nc[m];
      std::vector<double> e((size_t)nk[m] * nb);
      CK(cudaMemcpy(e.data(), c->eig.p, e.size() * 8, cudaMemcpyDeviceToHost));
      double gap = 50.0;
      for (int k = 0; k < nk[m]; ++k) gap = std::min(gap, e[(size_t)k * nb + nv[m]] - e[(size_t)k * nb + nv[m] - 1]);
      egap[m] = gap;
    }
  }
  return WTBG_OK;
}

int wtbg_eigsys(wtbg_ctx* ctx, int nk, const double* kpt, double* eig, double* vec, int* nocp) {
  if (!ctx || nk <= 0 || !kpt || !eig) return WTBG_ERR_ARG;
  if (ctx->w == 0) return set_err(ctx, WTBG_ERR_STATE, "eigsys: no model");
  if (int r = set_device(ctx)) return r;
  const int w = ctx->w;
  std::vector<double> kp(3 * (size_t)nk);
  for (int k = 0; k < nk; ++k)
    for (int c = 0; c < 3; ++c) kp[3 * k + c] = kpt[k + (size_t)nk * c];
  // scratch only within this call (the BSE state of the context is not touched)
  const size_t b_kpt = kp.size() * 8, b_eig = (size_t)nk * w * 8, b_int = (size_t)nk * 4;
  ENSURE(ctx->tmp, b_kpt + b_eig + 2 * b_int + 1024);
  ENSURE(ctx->ws, (size_t)nk * w * w * 16);
  char* base = ctx->tmp.as<char>();
  double* dk = reinterpret_cast<double*>(base);
  double* de = reinterpret_cast<double*>(base + (b_kpt + 255) / 256 * 256);
  int* dn = reinterpret_cast<int*>(base + (b_kpt + 255) / 256 * 256 + (b_eig + 255) / 256 * 256);
  int* ds = dn + nk;
  Timer t(ctx);
  CK(cudaMemcpyAsync(dk, kp.data(), b_kpt, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(ds, 0, b_int, ctx->stream));
  if (int r = launch_eigsys_all(ctx, nk, dk, de, ctx->ws.as<double2>(), dn, ds)) return r;
  if (int r = t.stop()) return r;
  std::vector<int> st(nk);
  CK(cudaMemcpy(st.data(), ds, b_int, cudaMemcpyDeviceToHost));
  for (int k = 0; k < nk; ++k)
    if (st[k] == 1) return set_err(ctx, WTBG_ERR_NOCONV, "eigsys: Jacobi did not converge at k-point " + std::to_string(k + 1));
  std::vector<double> e((size_t)nk * w);
  CK(cudaMemcpy(e.data(), de, b_eig, cudaMemcpyDeviceToHost));
  for (int k = 0; k < nk; ++k)
    for (int b = 0; b < w; ++b) eig[k + (size_t)nk * b] = e[(size_t)k * w + b];
  if (nocp) CK(cudaMemcpy(nocp, dn, b_int, cudaMemcpyDeviceToHost));
  if (vec) {
    std::vector<double2> u((size_t)nk * w * w);
    CK(cudaMemcpy(u.data(), ctx->ws.p, u.size() * 16, cudaMemcpyDeviceToHost));
    // vec(k, n, m): k fastest, then band n, then component m (the reference's autovetores per k)
    for (int k = 0; k < nk; ++k)
      for (int n = 0; n < w; ++n)
        for (int m = 0; m < w; ++m) {
          const double2 v = u[((size_t)k * w + n) * w + m];
          const size_t o = k + (size_t)nk * (n + (size_t)w * m);
          vec[2 * o] = v.x;
          vec[2 * o + 1] = v.y;
        }
  }
  return WTBG_OK;
}

int wtbg_berry(wtbg_ctx* ctx, int nk, const double* kpt, double gamma, double degtol, double* out) {
  if (!ctx || nk <= 0 || !kpt || !out) return WTBG_ERR_ARG;
  if (ctx->w == 0) return set_err(ctx, WTBG_ERR_STATE, "berry: no model");
  if (int r = set_device(ctx)) return r;
  const int w = ctx->w;
  std::vector<double> kp(3 * (size_t)nk);
  for (int k = 0; k < nk; ++k)
    for (int c = 0; c < 3; ++c) kp[3 * k + c] = kpt[k + (size_t)nk * c];
  // scratch only within this call (the BSE state of the context is not touched)
  const size_t b_kpt = kp.size() * 8, b_eig = (size_t)nk * w * 8, b_int = (size_t)nk * 4, b_out = (size_t)nk * 6 * 8;
  const size_t o_eig = (b_kpt + 255) / 256 * 256, o_int = o_eig + (b_eig + 255) / 256 * 256;
  const size_t o_out = o_int + (2 * b_int + 255) / 256 * 256;
  ENSURE(ctx->tmp, o_out + b_out + 256);
  ENSURE(ctx->ws, (size_t)nk * w * w * 16);
  char* base = ctx->tmp.as<char>();
  double* dk = reinterpret_cast<double*>(base);
  double* de = reinterpret_cast<double*>(base + o_eig);
  int* dn = reinterpret_cast<int*>(base + o_int);
  int* ds = dn + nk;
  double* dout = reinterpret_cast<double*>(base + o_out);
  Timer t(ctx);
  CK(cudaMemcpyAsync(dk, kp.data(), b_kpt, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(ds, 0, b_int, ctx->stream));
  if (int r = launch_eigsys_all(ctx, nk, dk, de, ctx->ws.as<double2>(), dn, ds)) return r;
  if (int r = launch_berry(ctx, nk, dk, de, ctx->ws.as<double2>(), dn, gamma, degtol, dout)) return r;
  if (int r = t.stop()) return r;
  std::vector<int> st(nk);
  CK(cudaMemcpy(st.data(), ds, b_int, cudaMemcpyDeviceToHost));
  for (int k = 0; k < nk; ++k)
    if (st[k] == 1) return set_err(ctx, WTBG_ERR_NOCONV, "berry: Jacobi did not converge at k-point " + std::to_string(k + 1));
  CK(cudaMemcpy(out, dout, b_out, cudaMemcpyDeviceToHost));
  return WTBG_OK;
}

int wtbg_sp_optbz(wtbg_ctx* ctx, int nk, const double* kpt, int nv, int nc, double sme, double* out) {
  if (!ctx || nk <= 0 || !kpt || !out || nv < 1 || nc < 1) return WTBG_ERR_ARG;
  if (ctx->w == 0) return set_err(ctx, WTBG_ERR_STATE, "opt_bz: no model");
  if (int r = set_device(ctx)) return r;
  const int w = ctx->w;
  std::vector<double> kp(3 * (size_t)nk);
  for (int k = 0; k < nk; ++k)
    for (int c = 0; c < 3; ++c) kp[3 * k + c] = kpt[k + (size_t)nk * c];
  const size_t b_kpt = kp.size() * 8, b_eig = (size_t)nk * w * 8, b_int = (size_t)nk * 4, b_out = (size_t)nk * 5 * 8;
  const size_t o_eig = (b_kpt + 255) / 256 * 256, o_int = o_eig + (b_eig + 255) / 256 * 256;
  const size_t o_out = o_int + (2 * b_int + 255) / 256 * 256;
  ENSURE(ctx->tmp, o_out + b_out + 256);
  ENSURE(ctx->ws, (size_t)nk * w * w * 16);
  char* base = ctx->tmp.as<char>();
  double* dk = reinterpret_cast<double*>(base);
  double* de = reinterpret_cast<double*>(base + o_eig);
  int* dn = reinterpret_cast<int*>(base + o_int);
  int* ds = dn + nk;
  double* dout = reinterpret_cast<double*>(base + o_out);
  Timer t(ctx);
  CK(cudaMemcpyAsync(dk, kp.data(), b_kpt, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(ds, 0, b_int, ctx->stream));
  if (int r = launch_eigsys_all(ctx, nk, dk, de, ctx->ws.as<double2>(), dn, ds)) return r;
  if (int r = launch_optbz(ctx, nk, nv, nc, dk, de, ctx->ws.as<double2>(), dn, sme, dout, ds)) return r;
  if (int r = t.stop()) return r;
  std::vector<int> st(nk);
  CK(cudaMemcpy(st.data(), ds, b_int, cudaMemcpyDeviceToHost));
  for (int k = 0; k < nk; ++k) {
    if (st[k] == 1) return set_err(ctx, WTBG_ERR_NOCONV, "opt_bz: Jacobi did not converge at k-point " + std::to_string(k + 1));
    if (st[k] == 4)
      return set_err(ctx, WTBG_ERR_BANDWINDOW,
                     "opt_bz: fewer than nc*nv band pairs at k-point " + std::to_string(k + 1) +
                         " (the valence range ends at the first k-point's nocp)");
  }
  CK(cudaMemcpy(out, dout, b_out, cudaMemcpyDeviceToHost));
  return WTBG_OK;
}

int wtbg_dos(wtbg_ctx* ctx, long long ndim, const double* etb, const double* weights, int ncol, long long nkpt,
             int nw, const double* en, double sme, double* out) {
  if (!ctx || ndim <= 0 || !etb || !weights || !en || !out || nw <= 0 || nkpt <= 0 || !(sme > 0))
    return WTBG_ERR_ARG;
  if (ncol < 1 || ncol > 4) return set_err(ctx, WTBG_ERR_ARG, "dos: 1 to 4 weight columns");
  if (int r = set_device(ctx)) return r;
  const size_t b_e = (size_t)ndim * 8, b_w = (size_t)ndim * ncol * 8, b_en = (size_t)nw * 8,
               b_o = (size_t)nw * ncol * 8;
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  ENSURE(ctx->tmp2, up(b_e) + up(b_w) + up(b_en) + up(b_o));
  char* base = ctx->tmp2.as<char>();
  double* d_e = reinterpret_cast<double*>(base);
  double* d_w = reinterpret_cast<double*>(base + up(b_e));
  double* d_en = reinterpret_cast<double*>(base + up(b_e) + up(b_w));
  double* d_o = reinterpret_cast<double*>(base + up(b_e) + up(b_w) + up(b_en));
  Timer t(ctx);
  CK(cudaMemcpyAsync(d_e, etb, b_e, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(d_w, weights, b_w, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(d_en, en, b_en, cudaMemcpyHostToDevice, ctx->stream));
  if (int r = launch_dos(ctx, d_e, d_w, ndim, ncol, d_en, nw, sme, nkpt, d_o)) return r;
  CK(cudaMemcpyAsync(out, d_o, b_o, cudaMemcpyDeviceToHost, ctx->stream));
  return t.stop();
}

int wtbg_set_temperature(wtbg_ctx* ctx, int on, double temp) {
  if (!ctx || on < 0 || on > 1 || !(temp >= 0.0)) return WTBG_ERR_ARG;
  ctx->temp_on = on;
  ctx->temp = temp;
  return WTBG_OK;
}

int wtbg_set_precision(wtbg_ctx* ctx, int mode) {
  if (!ctx || mode < 0 || mode > 1) return WTBG_ERR_ARG;
  if (int r = set_device(ctx)) return r;
  if (mode == 1) {
    ENSURE(ctx->pErr, 16);
    CK(cudaMemsetAsync(ctx->pErr.p, 0, 16, ctx->stream));
  }
  if (mode != ctx->prec) {
    // bands, velocities and matrix of the other form are not reused
    ctx->have_bands = ctx->have_velocity = ctx->have_matrix = ctx->have_solution = false;
    ctx->fast_ready = false;
  }
  ctx->prec = mode;
  return WTBG_OK;
}

int wtbg_set_fast_product(wtbg_ctx* ctx, int mode) {
  if (!ctx || mode < 0 || mode > 1) return WTBG_ERR_ARG;
  ctx->fast_mode = mode;
  return WTBG_OK;
}

int wtbg_bse_apply(wtbg_ctx* ctx, int m, const double* X, double* Y) {
  if (!ctx || !X || !Y || m < 1) return WTBG_ERR_ARG;
  if (!ctx->have_matrix) return set_err(ctx, WTBG_ERR_STATE, "bse_apply: call wtbg_bse_build first");
  if (int r = set_device(ctx)) return r;
  const long long N = ctx->N;
  const int mp = (m + 7) / 8 * 8;
  Timer t(ctx);
  ENSURE(ctx->tmp, (size_t)N * mp * 16);
  ENSURE(ctx->tmp2, (size_t)N * mp * 16);
  double2* dX = ctx->tmp.as<double2>();
  double2* dY = ctx->tmp2.as<double2>();
  CK(cudaMemsetAsync(dX, 0, (size_t)N * mp * 16, ctx->stream));
  CK(cudaMemcpyAsync(dX, X, (size_t)N * m * 16, cudaMemcpyHostToDevice, ctx->stream));
  if (ctx->fast_mode) {
    if (int r = run_fastprod(ctx, dX, (int)N, m, dY, (int)N)) return r;
    if (int r = fast_check(ctx)) return r;
  } else {
    for (int c = 0; c < mp; c += 8)
      if (int r = run_hemm_narrow(ctx, dX + (long long)c * N, (int)N, 8, dY + (long long)c * N, (int)N)) return r;
  }
  if (int r = t.stop()) return r;
  CK(cudaMemcpy(Y, dY, (size_t)N * m * 16, cudaMemcpyDeviceToHost));
  return WTBG_OK;
}

int wtbg_bse_spectrum_fast(wtbg_ctx* ctx, int nsteps, int dtfull, int cpol, double e1, double emax, const int* ngrid,
                           double vcell3d, double ebse0, double ebsef, double numbse, double sme, int renorm,
                           double spinf, double* omega, float* eps) {
  if (!ctx || !ngrid || !omega || !eps) return WTBG_ERR_ARG;
  if (!ctx->have_matrix) return set_err(ctx, WTBG_ERR_STATE, "bse_spectrum_fast: call wtbg_bse_build first");
  if (!ctx->have_velocity) return set_err(ctx, WTBG_ERR_STATE, "bse_spectrum_fast: call wtbg_velocity first");
  if (ctx->temp_on) return set_err(ctx, WTBG_ERR_UNSUPPORTED, "bse_spectrum_fast: no temperature form");
  const int nw = (int)numbse;
  if (nsteps < 2 || nw < 2) return set_err(ctx, WTBG_ERR_ARG, "bse_spectrum_fast: bad sizes");
  if (int r = set_device(ctx)) return r;
  // chains: x, y, z [, x+y, x-y, x+z, x-z, y+z, y-z] [, sp, sm]
  std::vector<int> codes = {0, 1, 2};
  if (dtfull)
    for (int k = 5; k <= 10; ++k) codes.push_back(k);
  const int isp = (int)codes.size();
  if (cpol) {
    codes.push_back(3);
    codes.push_back(4);
  }
  // outputs (kind, chain): 8 components, absent ones point at chain 0 with kind 2 (zero)
  std::vector<int> oc(16);
  auto put = [&](int o, int kind, int ch) {
    oc[2 * o] = kind;
    oc[2 * o + 1] = ch;
  };
  put(0, 0, 0);
  put(1, 0, 1);
  put(2, 0, 2);
  if (dtfull) {
    put(3, 1, 3);
    put(4, 1, 5);
    put(5, 1, 7);
  } else {
    put(3, 1, 0);
    put(4, 1, 0);
    put(5, 1, 0);
  }
  if (cpol) {
    put(6, 0, isp);
    put(7, 0, isp + 1);
  } else {
    put(6, 1, 0);
    put(7, 1, 0);
  }
  const long long N = ctx->N;
  const double eta = sme + 10.0 * ((emax - e1) / (double)N);
  Timer t(ctx);
  std::vector<double> al, be, n2;
  if (int r = run_haydock(ctx, nsteps, (int)codes.size(), codes.data(), al, be, n2)) return r;
  if (ctx->fast_mode)
    if (int r = fast_check(ctx)) return r;
  ENSURE(ctx->sp_om, (size_t)nw * 8 + (size_t)nw * 16 * 4 + 64);
  double* dom = ctx->sp_om.as<double>();
  float* deps = reinterpret_cast<float*>(dom + nw);
  if (int r = run_haydock_spectrum(ctx, nsteps, (int)codes.size(), al.data(), be.data(), n2.data(), 8, oc.data(), ngrid,
                                   vcell3d, ebse0, ebsef, numbse, eta, e1, renorm, spinf, dom, deps))
    return r;
  CK(cudaMemcpyAsync(omega, dom, (size_t)nw * 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(eps, deps, (size_t)nw * 16 * 4, cudaMemcpyDeviceToHost, ctx->stream));
  if (int r = t.stop()) return r;
  // components that were not requested (kind 1 on chain 0 with chain 0 - chain 1 is not zero):
  // zero them explicitly
  for (int o = 3; o < 8; ++o) {
    const bool want = (o < 6) ? dtfull : cpol;
    if (!want)
      for (int j = 0; j < nw; ++j) {
        eps[(size_t)j + (size_t)nw * (0 + 2 * o)] = 0.0f;
        eps[(size_t)j + (size_t)nw * (1 + 2 * o)] = 0.0f;
      }
  }
  return WTBG_OK;
}

int wtbg_bse_eigvecs(wtbg_ctx* ctx, int n0, int n1, double* A) {
  if (!ctx || !A) return WTBG_ERR_ARG;
  if (!ctx->have_solution || ctx->csize_host.empty())
    return set_err(ctx, WTBG_ERR_STATE, "bse_eigvecs: call wtbg_bse_solve (with act) first");
  if (n0 < 1 || n1 < n0 || n1 > ctx->N) return set_err(ctx, WTBG_ERR_ARG, "bse_eigvecs: bad range");
  if (int r = set_device(ctx)) return r;
  const long long N = ctx->N;
  ENSURE(ctx->yv, (size_t)N * 32 * 16);
  double ms = 0.0;
  for (int a0 = n0; a0 <= n1; a0 += 32) {
    const int a1 = (a0 + 31 < n1) ? a0 + 31 : n1;
    const int nvec = a1 - a0 + 1;
    Timer t(ctx);
    if (int r = run_eigvecs(ctx, a0, a1, ctx->yv.as<double2>())) return r;
    if (int r = t.stop()) return r;
    ms += ctx->last_ms;
    CK(cudaMemcpy(A + 2 * (size_t)N * (a0 - n0), ctx->yv.p, (size_t)N * nvec * 16, cudaMemcpyDeviceToHost));
  }
  ctx->last_ms = ms;
  return WTBG_OK;
}

int wtbg_spectrum(wtbg_ctx* ctx, int n, int ncomp, const double* ebse, const double* fosc, const int* rtype,
                  const int* ngrid, double vcell3d, double ebse0, double ebsef, double numbse, double sme, int renorm,
                  double spinf, double* omega, float* eps) {
  if (!ctx || !ebse || !fosc || !rtype || !ngrid || !omega || !eps) return WTBG_ERR_ARG;
  const int nw = (int)numbse;
  if (n <= 0 || nw < 2 || ncomp < 1 || ncomp > 8) return set_err(ctx, WTBG_ERR_ARG, "spectrum: bad sizes");
  if (int r = set_device(ctx)) return r;
  ENSURE(ctx->sp_in, (size_t)n * (ncomp + 1) * 8);
  ENSURE(ctx->sp_om, (size_t)nw * 8 + (size_t)nw * 2 * ncomp * 4 + 64);
  double* de = ctx->sp_in.as<double>();
  double* df = de + n;
  double* dom = ctx->sp_om.as<double>();
  float* deps = reinterpret_cast<float*>(dom + nw);
  Timer t(ctx);
  CK(cudaMemcpyAsync(de, ebse, (size_t)n * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(df, fosc, (size_t)n * ncomp * 8, cudaMemcpyHostToDevice, ctx->stream));
  if (int r = launch_spectrum(ctx, n, ncomp, de, df, rtype, ngrid, vcell3d, ebse0, ebsef, numbse, sme, renorm, spinf,
                              dom, deps))
    return r;
  CK(cudaMemcpyAsync(omega, dom, (size_t)nw * 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(eps, deps, (size_t)nw * 2 * ncomp * 4, cudaMemcpyDeviceToHost, ctx->stream));
  if (int r = t.stop()) return r;
  return WTBG_OK;
}

int wtbg_bse_build_q(wtbg_ctx* ctx, int nk, const double* kptq, const double* q4, const wtbg_coulomb* p) {
  if (!ctx || !kptq || !q4 || !p) return WTBG_ERR_ARG;
  if (!ctx->have_bands || nk != ctx->nk) return set_err(ctx, WTBG_ERR_STATE, "bse_q: call wtbg_bands on the k-mesh first");
  if (int r = set_device(ctx)) return r;
  const int nb = ctx->nv + ctx->nc, w = ctx->w;
  const long long N = ctx->N;
  std::vector<double> kq(3 * (size_t)nk);
  for (int k = 0; k < nk; ++k)
    for (int c = 0; c < 3; ++c) kq[3 * k + c] = kptq[k + (size_t)nk * c];
  ENSURE(ctx->kptq, kq.size() * 8);
  ENSURE(ctx->eigq, (size_t)nk * nb * 8);
  ENSURE(ctx->Uq, (size_t)nk * nb * w * 16);
  ENSURE(ctx->nocpq, (size_t)nk * 4);
  ENSURE(ctx->H, (size_t)N * N * 16);
  Timer t(ctx);
  CK(cudaMemcpyAsync(ctx->kptq.p, kq.data(), kq.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
  if (int r = launch_bands(ctx, true)) return r;
  if (int r = check_kstat(ctx, nk)) return r;
  if (int r = check_gemm_err(ctx)) return r;
  if (int r = launch_bse_build(ctx, p, q4)) return r;
  if (int r = t.stop()) return r;
  if (int r = check_gemm_err(ctx)) return r;
  ctx->have_matrix = true;
  ctx->fast_ready = false;
  ctx->have_solution = false;
  return WTBG_OK;
}

int wtbg_bse_q_eigenvalues(wtbg_ctx* ctx, int nk, const double* kptq, const double* q4, const wtbg_coulomb* p,
                           double* W) {
  if (!ctx || !kptq || !q4 || !p || !W) return WTBG_ERR_ARG;
  if (int r = wtbg_bse_build_q(ctx, nk, kptq, q4, p)) return r;
  const long long N = ctx->N;
  Timer t(ctx);
  const bool hv = ctx->have_velocity;
  ctx->have_velocity = false;   // eigenvalues only: g not needed
  int r = run_tridiagonalise(ctx);
  ctx->have_velocity = hv;
  if (r) return r;
  if ((r = run_tridiagonal_solve(ctx, 0, 0, false))) return r;
  if ((r = t.stop())) return r;
  ctx->have_matrix = false;
  ctx->fast_ready = false;
  ctx->have_solution = false;
  memcpy(W, ctx->lam_host.data(), (size_t)N * 8);
  return WTBG_OK;
}

// Tridiagonalises the current matrix through one captured CUDA graph of the whole
// column loop. The first call for a given N (or after any work buffer moved) runs eagerly,
// which also sizes the buffers and autotunes the mat-vec chunk; the next call captures the
// launch sequence into a graph, and every later call replays it. The graph reads the matrix
// and writes the tridiagonal through the context's buffers, so it serves every Q of a batch.
static int tridiagonalise_graph(wtbg_ctx* ctx) {
  if (use_two_stage(ctx)) return run_tridiagonalise(ctx);   // a few launches per panel: no graph needed
  auto signature = [ctx]() {
    return std::vector<const void*>{ctx->H.p,     ctx->d.p,    ctx->e.p,     ctx->tau.p,  ctx->g.p,
                                     ctx->Wp.p,    ctx->slots.p, ctx->part.p, ctx->scal.p, ctx->h.p,
                                     ctx->fdeh.p,  (const void*)(intptr_t)ctx->N,
                                     (const void*)(intptr_t)ctx->hemv_hs,
                                     (const void*)(intptr_t)(ctx->have_velocity ? 1 + ctx->temp_on : 0)};
  };
  if (ctx->profiling) return run_tridiagonalise(ctx);   // per-launch events need host syncs
  std::vector<const void*> sig = signature();
  if (ctx->tri_exec && sig == ctx->tri_sig) {
    CK(cudaGraphLaunch(ctx->tri_exec, ctx->stream));
    WTBG_COUNT(ctx, ctx->tri_launches);
    return 0;
  }
  if (ctx->tri_exec) {
    cudaGraphExecDestroy(ctx->tri_exec);
    ctx->tri_exec = nullptr;
  }
  if (sig != ctx->tri_sig) {
    if (int r = run_tridiagonalise(ctx)) return r;
    ctx->tri_sig = signature();
    return 0;
  }
  cudaGraph_t graph = nullptr;
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  const long long l0 = ctx->stats.launches;
  const int r = run_tridiagonalise(ctx);
  const cudaError_t ec = cudaStreamEndCapture(ctx->stream, &graph);
  const long long nl = ctx->stats.launches - l0;
  ctx->stats.launches = l0;
  if (r) {
    if (graph) cudaGraphDestroy(graph);
    return r;
  }
  if (ec != cudaSuccess) return cuda_fail(ctx, ec, "cudaStreamEndCapture(tridiagonalise)");
  const cudaError_t ei = cudaGraphInstantiate(&ctx->tri_exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ei != cudaSuccess) {
    ctx->tri_exec = nullptr;
    return cuda_fail(ctx, ei, "cudaGraphInstantiate(tridiagonalise)");
  }
  if (signature() != sig) return set_err(ctx, WTBG_ERR_STATE, "tridiagonalise: work buffers moved during capture");
  ctx->tri_launches = nl;
  CK(cudaGraphLaunch(ctx->tri_exec, ctx->stream));
  WTBG_COUNT(ctx, nl);
  return 0;
}

// Q points of the two-stage path in groups of up to kQGroup: stage 1 of each Q into its own band
// slot (the N x N matrix buffer is reused), one bulge-chasing launch for the group's bands, then
// the eigenvalues of each tridiagonal form.  ms_q gets the group's device time divided evenly.
constexpr int kQGroup = 64;
static int q_group_two_stage(wtbg_ctx* ctx, int nk, int g0, int gn, const double* kptq, const double* q4,
                             const wtbg_coulomb* p, double* W, double* ms_q) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  int r = 0;
  long long N = 0;
  const bool hv = ctx->have_velocity;
  cudaEventRecord(e0, ctx->stream);
  for (int i = 0; i < gn && !r; ++i) {
    const int iq = g0 + i;
    if ((r = wtbg_bse_build_q(ctx, nk, kptq + (size_t)iq * nk * 3, q4 + (size_t)iq * 4, p))) break;
    if (i == 0) {
      N = ctx->N;
      if ((r = two_stage_group_begin(ctx, gn))) break;
    }
    ctx->have_velocity = false;
    r = two_stage_group_add(ctx, i);
    ctx->have_velocity = hv;
  }
  double* dd = nullptr;
  double* ee = nullptr;
  if (!r) r = two_stage_group_finish(ctx, gn, &dd, &ee);
  for (int i = 0; i < gn && !r; ++i) {
    cudaError_t ce = cudaMemcpyAsync(ctx->d.p, dd + (size_t)i * N, (size_t)N * 8, cudaMemcpyDeviceToDevice, ctx->stream);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(ctx->e.p, ee + (size_t)i * N, (size_t)N * 8, cudaMemcpyDeviceToDevice, ctx->stream);
    if (ce != cudaSuccess) {
      r = cuda_fail(ctx, ce, "Q group: tridiagonal copy");
      break;
    }
    if ((r = run_tridiagonal_solve(ctx, 0, 0, false))) break;
    memcpy(W + (size_t)(g0 + i) * N, ctx->lam_host.data(), (size_t)N * 8);
  }
  if (!r) {
    cudaEventRecord(e1, ctx->stream);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms_q)
      for (int i = 0; i < gn; ++i) ms_q[g0 + i] = ms / gn;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return r;
}

int wtbg_bse_q_batch(wtbg_ctx* ctx, int nk, int nq, const double* kptq, const double* q4, const wtbg_coulomb* p,
                     int use_graph, double* W, double* ms_q) {
  if (!ctx || !kptq || !q4 || !p || !W || nq < 0) return WTBG_ERR_ARG;
  if (nq == 0) return WTBG_OK;
  if (!ctx->have_bands) return set_err(ctx, WTBG_ERR_STATE, "bse_q_batch: call wtbg_bands first");
  const bool hv = ctx->have_velocity;
  int r = 0;
  {
    // the reduction is decided by N = nk nc nv, the same for every Q
    const long long N0 = ctx->N;
    ctx->N = (long long)nk * ctx->nc * ctx->nv;
    const bool two = use_two_stage(ctx);
    ctx->N = N0;
    if (two) {
      for (int g0 = 0; g0 < nq && !r; g0 += kQGroup)
        r = q_group_two_stage(ctx, nk, g0, std::min(kQGroup, nq - g0), kptq, q4, p, W, ms_q);
      ctx->have_velocity = hv;
      ctx->have_matrix = false;
      ctx->fast_ready = false;
      ctx->have_solution = false;
      return r ? r : WTBG_OK;
    }
  }
  for (int iq = 0; iq < nq && !r; ++iq) {
    if ((r = wtbg_bse_build_q(ctx, nk, kptq + (size_t)iq * nk * 3, q4 + (size_t)iq * 4, p))) break;
    const double ms_build = ctx->last_ms;
    const long long N = ctx->N;
    Timer t(ctx);
    ctx->have_velocity = false;   // eigenvalues only: g not needed
    r = use_graph ? tridiagonalise_graph(ctx) : run_tridiagonalise(ctx);
    ctx->have_velocity = hv;
    if (r) break;
    if ((r = run_tridiagonal_solve(ctx, 0, 0, false))) break;
    if ((r = t.stop())) break;
    memcpy(W + (size_t)iq * N, ctx->lam_host.data(), (size_t)N * 8);
    if (ms_q) ms_q[iq] = ms_build + ctx->last_ms;
  }
  ctx->have_velocity = hv;
  ctx->have_matrix = false;
  ctx->fast_ready = false;
  ctx->have_solution = false;
  return r ? r : WTBG_OK;
}

}  // extern "C"
