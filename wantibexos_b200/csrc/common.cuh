// Shared definitions for libwtbgpu.so (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/wtbgpu.h"

#define WTBG_MAX_W 256         // largest orbital count of the per-k eigensolver (one thread per band)
#define WTBG_HEMV_TILE 64      // tile edge of the Hermitian matrix-vector kernel
#define WTBG_PANEL 32          // Householder panel width of the tridiagonalisation

// Device buffer that only grows.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

struct wtbg_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = 0.0;
  std::string err;

  // model (hamiltonian_input_variables)
  int w = 0, nvec = 0;
  double rlat[9] = {0};   // row-major rlat[i*3+c] = a_i component c
  double efermi = 0.0, scs = 0.0;
  DevBuf HR;      // [nvec][n][m] double2 : H_mn(R)
  DevBuf Rcart;   // [nvec][3] double : Cartesian R in the reference evaluation order
  DevBuf Rf32;    // [nvec][3] double : float32-rounded Cartesian R (velocity prefactor)
  DevBuf invdeg;  // [nvec] double : 1/deg(R)
  DevBuf isR0;    // [nvec] int

  // k-mesh bands
  int nk = 0, nv = 0, nc = 0;
  DevBuf kpt;     // [nk][3]
  DevBuf eig;     // [nk][nc+nv]
  DevBuf U;       // [nk][nc+nv][w] double2
  DevBuf nocp;    // [nk] int
  DevBuf kstat;   // [nk] int (per-k status)
  bool have_bands = false;

  // k+Q bands (exciton band structure)
  DevBuf kptq, eigq, Uq, nocpq;

  // velocity
  DevBuf h;       // [5][N] double2
  bool have_velocity = false;

  // BSE matrix and dense-solve state
  long long N = 0;
  DevBuf H;       // N*N double2, lower triangle column-major
  bool have_matrix = false;
  DevBuf d, e, tau, g;     // tridiagonal, reflector scalars, g = Q^T h  ([5][N] double2)
  DevBuf Wp;               // panel W (N x PANEL) double2
  DevBuf slots;            // hemv partials
  DevBuf part;             // small partial-reduction area
  DevBuf scal;             // per-column scalars
  DevBuf yv;               // hemv result
  DevBuf lam;              // eigenvalues
  DevBuf bgrid;            // coarse multisection grid: points and Sturm counts
  DevBuf ws;               // inverse-iteration workspace
  DevBuf act;              // oscillator strengths [8][N]
  DevBuf zsel;             // selected tridiagonal eigenvectors (for eigvecs)
  DevBuf csz;              // cluster size per eigenvalue index (leaders), 0 otherwise
  std::vector<double> lam_host;
  std::vector<int> csize_host;
  double tnorm = 0.0;
  bool have_solution = false;

  // spectrum
  DevBuf sp_in, sp_out, sp_om;

  // misc
  DevBuf tmp, tmp2, istat;
  DevBuf gwork;   // per-CTA work areas of the per-k kernels for models too large for shared memory

  // counters
  // temperature BSE (BSET / BSET_BND): occupation factor f_v - f_c per basis state
  int temp_on = 0;
  double temp = 0.0;     // temperature used in the Fermi factors (0 is replaced as the reference does)
  DevBuf fdeh;           // [N] double
  int ng = 5;            // velocity vectors carried through the reduction (10 with temperature)

  // tridiagonalisation: autotuned mat-vec chunk, and the captured CUDA graph of the whole
  // reduction for Q batches (valid while N and the work buffers stay the same)
  int hemv_hs = 0;
  int nsm = 0;
  alignas(64) unsigned char tmH[128];   // CUtensorMap of H for the mat-vec (see prepare_hemv)
  const void* tmH_ptr = nullptr;
  long long tmH_n = 0;
  DevBuf triErr;                        // set by the mat-vec when a pipeline wait timed out
  // two-stage reduction (tridiag2.cu): mode 0 auto, 1 one-stage, 2 two-stage; which one ran last
  int tri_mode = 0;
  bool tri_two = false;
  int bulge_warp_mode = 0;   // stage 2: 0 = one CTA of four warps per sweep, 1 = one warp per sweep
  DevBuf t2V, t2X, t2D, t2G, t2T, t2P, t2AB, t2prog, t2de;
  cudaGraphExec_t tri_exec = nullptr;
  std::vector<const void*> tri_sig;
  long long tri_launches = 0;

  // precision form (0 = FP64; 1 = Fourier sums and band overlaps as 3-term split-BF16
  // tensor-core products with FP32 accumulation)
  int prec = 0;
  DevBuf pOpA, pOpB, pHk, pOc, pOv, pErr;

  // fast form: split-BF16 planes of the kernel matrix for the tensor-core product
  int fast_mode = 0;
  bool fast_ready = false;
  long long fast_ld = 0;
  int fast_mp = 0;
  DevBuf fA, fB, fY, fD, fErr;
  alignas(64) unsigned char tmA[128];   // CUtensorMap of the H planes
  alignas(64) unsigned char tmB[128];   // CUtensorMap of the X planes (current padded width)

  wtbg_stats stats{};
  int profiling = 0;
  std::vector<cudaEvent_t> evpool;   // event pairs for per-launch timing when profiling
};

// make sure the event pool holds at least n events
int ensure_events(wtbg_ctx* ctx, size_t n);

// launch accounting: count every kernel launch issued through a context
#define WTBG_COUNT(ctx, n) ((ctx)->stats.launches += (n))

// error handling
int set_err(wtbg_ctx* c, int code, const std::string& msg);
int cuda_fail(wtbg_ctx* c, cudaError_t e, const char* where);
int ensure(wtbg_ctx* c, DevBuf& b, size_t bytes);

#define CK(call)                                                  \
  do {                                                            \
    cudaError_t _e = (call);                                      \
    if (_e != cudaSuccess) return cuda_fail(ctx, _e, #call);      \
  } while (0)

#define CKL(where)                                                \
  do {                                                            \
    cudaError_t _e = cudaGetLastError();                          \
    if (_e != cudaSuccess) return cuda_fail(ctx, _e, where);      \
  } while (0)

#define ENSURE(buf, bytes)                                        \
  do {                                                            \
    int _r = ensure(ctx, (buf), (bytes));                         \
    if (_r) return _r;                                            \
  } while (0)

// ---- complex helpers (double2 = re, im)
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // conj(a)*b
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) {
  return make_double2(a.x * s, a.y * s);
}
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// ---- kernel launchers (implemented in the .cu files)
int launch_bands(wtbg_ctx* ctx, bool q_mesh);
int launch_velocity(wtbg_ctx* ctx, double eta_f32);
int launch_sp_table(wtbg_ctx* ctx, float* d_out);
int launch_bse_build(wtbg_ctx* ctx, const wtbg_coulomb* p, const double* q4);
int run_tridiagonalise(wtbg_ctx* ctx);
int run_tridiagonal_solve(wtbg_ctx* ctx, int dtfull, int cpol, bool vectors);
int run_eigvecs(wtbg_ctx* ctx, int n0, int n1, double2* d_out);
int run_haydock(wtbg_ctx* ctx, int K, int ncomp, const int* codes, std::vector<double>& alpha, std::vector<double>& beta,
                std::vector<double>& norm2);
int run_haydock_spectrum(wtbg_ctx* ctx, int K, int nchain, const double* alpha, const double* beta, const double* norm2,
                         int nout, const int* ocode, const int* ngrid, double vcell3d, double ebse0, double ebsef,
                         double numbse, double eta, double e1, int renorm, double spinf, double* d_om, float* d_eps);
// CUDA-event timing of one C-ABI call on the context's stream (sets last_ms)
struct Timer {
  wtbg_ctx* c;
  explicit Timer(wtbg_ctx* ctx) : c(ctx) { cudaEventRecord(c->ev0, c->stream); }
  int stop() {
    cudaEventRecord(c->ev1, c->stream);
    cudaError_t e = cudaEventSynchronize(c->ev1);
    if (e != cudaSuccess) return cuda_fail(c, e, "stream");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->last_ms = ms;
    return 0;
  }
};


inline int set_device(wtbg_ctx* ctx) {
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  return 0;
}


int launch_bands_batch(wtbg_ctx* const* ctxs, int nmod);
int launch_eigsys_all(wtbg_ctx* ctx, int nk, const double* d_kpt, double* d_eig, double2* d_U, int* d_nocp,
                      int* d_kstat);
int launch_berry(wtbg_ctx* ctx, int nk, const double* d_kpt, const double* d_eig, const double2* d_U, const int* d_nocp,
                 double gamma, double degtol, double* d_out);
int launch_optbz(wtbg_ctx* ctx, int nk, int nv, int nc, const double* d_kpt, const double* d_eig, const double2* d_U,
                 const int* d_nocp, double sme, double* d_out, int* d_kstat);
int launch_dos(wtbg_ctx* ctx, const double* d_etb, const double* d_w, long long ndim, int ncol, const double* d_en,
               int nw, double sme, long long nkpt, double* d_out);
int autotune_hemv(wtbg_ctx* ctx, int* hs_out);
int run_backtransform2(wtbg_ctx* ctx, double2* X, int nvec);
int two_stage_group_begin(wtbg_ctx* ctx, int nq);
int two_stage_group_add(wtbg_ctx* ctx, int slot);
int two_stage_group_finish(wtbg_ctx* ctx, int nq, double** dd, double** ee);
bool use_two_stage(wtbg_ctx* ctx);
// C^T (N x M, ldc) (+)= A (M x K, lda) B (N x K, ldb)^T, bf16 operands, FP32 accumulation on the
// tensor cores (tcgen05); err is a device flag set when a pipeline wait times out
int gemm_bf16(wtbg_ctx* ctx, int* err, const __nv_bfloat16* A, long long lda, int M, int K, const __nv_bfloat16* B,
              long long ldb, int N, float* C, long long ldc, bool clear);
int check_gemm_err(wtbg_ctx* ctx);

// 3-term split of a double into bf16 hi + lo (x ~ hi + lo to about 16 significant bits)
__device__ __forceinline__ void split_bf16(double x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __double2bfloat16(x);
  lo = __double2bfloat16(x - (double)__bfloat162float(hi));
}
// One operand row of the 3-term product sum_s a_s b_s ~ ah.bh + ah.bl + al.bh from its real
// values: the A side is stored [hi | hi | lo], the B side [hi | lo | hi] (K = 3 * width)
__device__ __forceinline__ void put_split_row(__nv_bfloat16* row, int width, int s, double x, bool a_side) {
  __nv_bfloat16 hi, lo;
  split_bf16(x, hi, lo);
  row[s] = hi;
  row[width + s] = a_side ? hi : lo;
  row[2 * width + s] = a_side ? lo : hi;
}
int ensure_fdeh(wtbg_ctx* ctx, bool q_mesh);
int fill_g_vectors(wtbg_ctx* ctx, double2* g);
int run_fast_setup(wtbg_ctx* ctx);
int run_fastprod(wtbg_ctx* ctx, const double2* X, int ldx, int m, double2* Y, int ldy);
int run_hemm_narrow(wtbg_ctx* ctx, const double2* X, int ldx, int m, double2* Y, int ldy);
int fast_check(wtbg_ctx* ctx);
int run_davidson(wtbg_ctx* ctx, int nev, int nb, int largest, int max_iter, double tol, const double2* dX0, int dtfull,
                 int cpol, std::vector<double>& W, std::vector<double>& act, double2* dXout, int* iters, double* maxres);
int launch_spectrum(wtbg_ctx* ctx, int n, int ncomp, const double* d_e, const double* d_f, const int* rtype,
                    const int* ngrid, double vcell3d, double ebse0, double ebsef, double numbse, double sme,
                    int renorm, double spinf, double* d_om, float* d_eps);
