// Kernel (d): broadened dielectric function of the BSE spectrum.
//
// Reference: bsedielraw (subprograms/bse_diel-tool.f90:137-210) calling optdiel
// (subroutines/optics.f90:160-244), avgsme (:302-324) and imagrenorm (:327-390):
//   eta   = CSHIFT + 10 * sum_{i>=2}(E_i - E_{i-1}) / N          (summed in order)
//   c     = float32(180.90) / (float32(nk) * V_cell)
//   Re eps(w) = delta + c * sum_n f_n (E_n - w) / ((w - E_n)^2 + eta^2)
//   Im eps(w) =         c * sum_n f_n  eta      / ((w - E_n)^2 + eta^2)
//   then (RNMD) Im is zeroed below E_1 - float32(0.15) and shifted down by its value at
//   the next grid point (clamped at 0), and every value is written as real(spinf * x).
// One warp per photon energy reduces over the excitons with shuffles; the six tensor
// components share the two divisions of each (w, n) term.
#include <cstdio>
#include <map>
#include <mutex>

#include "common.cuh"

namespace {

__global__ void k_avgsme(const double* e, int n, double sme, double* eta_out) {
  // sequential, in the reference's order (one thread)
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int i = 1; i < n; ++i) s = s + e[i] - e[i - 1];
  *eta_out = 10.0 * (s / (double)n) + sme;
}

constexpr int kMaxComp = 8;

struct SpecRtype {
  int rt[kMaxComp];
};

template <int NCOMP>
__global__ void __launch_bounds__(256) k_spectrum(const double* __restrict__ E, const double* __restrict__ F, int n,
                                                  const double* __restrict__ eta_p, double ebse0, double ebsef,
                                                  double numbse, int nw, double caux, SpecRtype rt, double* om,
                                                  double* re, double* im) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= nw) return;
  const int j = warp + 1;
  const double w = ebse0 + (((ebsef - ebse0) * (j - 1)) / (numbse - 1.));
  const double eta = *eta_p;
  const double eta2 = eta * eta;
  double r[NCOMP], a[NCOMP];
#pragma unroll
  for (int c = 0; c < NCOMP; ++c) r[c] = a[c] = 0.0;
  for (int i = lane; i < n; i += 32) {
    const double e = E[i];
    const double eaux = ((w - e) * (w - e)) + eta2;
    const double d1 = (e - w) / eaux;
    const double d2 = eta / eaux;
#pragma unroll
    for (int c = 0; c < NCOMP; ++c) {
      const double f = F[(long long)c * n + i];
      r[c] += f * d1;
      a[c] += f * d2;
    }
  }
#pragma unroll
  for (int c = 0; c < NCOMP; ++c) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      r[c] += __shfl_xor_sync(0xffffffffu, r[c], o);
      a[c] += __shfl_xor_sync(0xffffffffu, a[c], o);
    }
  }
  if (lane == 0) {
    om[warp] = w;
#pragma unroll
    for (int c = 0; c < NCOMP; ++c) {
      const double delta = rt.rt[c] == 1 ? 1.0 : 0.0;
      re[(long long)c * nw + warp] = delta + (r[c] * caux);
      im[(long long)c * nw + warp] = a[c] * caux;
    }
  }
}

// imagrenorm per component + real(spinf*x) output, eps(nw,2,6)
__global__ void k_renorm_out(const double* E, const double* om, const double* re, double* im, int nw, int ncomp,
                             int renorm, double spinf, float* eps) {
  const int c = threadIdx.x;
  if (c >= ncomp) return;
  double* ic = im + (long long)c * nw;
  if (renorm) {
    const double aux = E[0] - (double)0.15f;
    if (!(aux <= 0.000)) {
      int ibegin = 1;
      for (int i = 1; i <= nw; ++i) {
        if (om[i - 1] <= aux) ibegin = i;
        else break;
      }
      const double aux3 = (ibegin < nw) ? ic[ibegin] : 0.0;   // dielf(ibegin+1,3)
      for (int i = 1; i <= ibegin; ++i) ic[i - 1] = 0.0;
      for (int i = ibegin + 1; i <= nw; ++i) {
        const double v = ic[i - 1] - aux3;
        ic[i - 1] = (v < 0.0) ? 0.0 : v;
      }
    }
  }
  for (int i = 0; i < nw; ++i) {
    eps[(long long)i + (long long)nw * (0 + 2 * c)] = (float)(spinf * re[(long long)c * nw + i]);
    eps[(long long)i + (long long)nw * (1 + 2 * c)] = (float)(spinf * ic[i]);
  }
}

}  // namespace

int launch_spectrum(wtbg_ctx* ctx, int n, int ncomp, const double* d_e, const double* d_f, const int* rtype,
                    const int* ngrid, double vcell3d, double ebse0, double ebsef, double numbse, double sme,
                    int renorm, double spinf, double* d_om, float* d_eps) {
  const int nw = (int)numbse;
  ENSURE(ctx->sp_out, (size_t)2 * kMaxComp * nw * 8 + 64);
  double* re = ctx->sp_out.as<double>();
  double* im = re + (size_t)ncomp * nw;
  double* eta = im + (size_t)ncomp * nw;
  SpecRtype rt{};
  for (int c = 0; c < ncomp; ++c) rt.rt[c] = rtype[c];
  const double baux = (double)(float)(ngrid[0] * ngrid[1] * ngrid[2]) * vcell3d;
  const double caux = (double)180.90f / (baux * 1.0);
  k_avgsme<<<1, 32, 0, ctx->stream>>>(d_e, n, sme, eta); WTBG_COUNT(ctx, 1);
  CKL("k_avgsme");
  const int threads = 256;
  const int blocks = (nw * 32 + threads - 1) / threads;
  switch (ncomp) {
#define WTBG_SPEC_CASE(K)                                                                                      \
  case K:                                                                                                      \
    k_spectrum<K><<<blocks, threads, 0, ctx->stream>>>(d_e, d_f, n, eta, ebse0, ebsef, numbse, nw, caux, rt,   \
                                                       d_om, re, im);                                          \
    break;
    WTBG_SPEC_CASE(1) WTBG_SPEC_CASE(2) WTBG_SPEC_CASE(3) WTBG_SPEC_CASE(4)
    WTBG_SPEC_CASE(5) WTBG_SPEC_CASE(6) WTBG_SPEC_CASE(7) WTBG_SPEC_CASE(8)
#undef WTBG_SPEC_CASE
    default: return set_err(ctx, WTBG_ERR_ARG, "spectrum: ncomp must be 1..8");
  }
  WTBG_COUNT(ctx, 1);
  CKL("k_spectrum");
  k_renorm_out<<<1, 32, 0, ctx->stream>>>(d_e, d_om, re, im, nw, ncomp, renorm, spinf, d_eps); WTBG_COUNT(ctx, 1);
  CKL("k_renorm_out");
  return 0;
}

// ---- DOS smearing (endos, subroutines/dos_subs.f90:102-152, with gaussian,
//      general_subs.f90:471-487): out[e][c] = (1/nkpt) sum_i w_c(i) g(en_e - etb_i),
//      g(x) = exp(-x^2 / (2 sme^2)) / (sme sqrt(2 pi)), pi = acos(-1.) in real(4).
namespace {
__global__ void k_dos(const double* etb, const double* w, long long ndim, int ncol, const double* en, int nw,
                      double sme, double caux, double* out) {
  const int e = blockIdx.x;
  if (e >= nw) return;
  const double pi32 = (double)3.14159274101257324f;
  const double norm = 1.0 / (sme * sqrt(2.0 * pi32));
  const double deno = 2.0 * sme * sme;
  const double x0 = en[e];
  __shared__ double red[8][4];
  double acc[4] = {0, 0, 0, 0};
  for (long long i = threadIdx.x; i < ndim; i += blockDim.x) {
    const double dx = x0 - etb[i];
    const double g = norm * exp(-1.0 * (dx * dx) / deno);
    for (int c = 0; c < ncol && c < 4; ++c) acc[c] += w[c * ndim + i] * g;
  }
  for (int c = 0; c < 4; ++c)
    for (int o = 16; o > 0; o >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
  if ((threadIdx.x & 31) == 0)
    for (int c = 0; c < 4; ++c) red[threadIdx.x >> 5][c] = acc[c];
  __syncthreads();
  if (threadIdx.x < ncol) {
    double s = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[k][threadIdx.x];
    out[(long long)threadIdx.x * nw + e] = s * caux;
  }
}
}  // namespace

int launch_dos(wtbg_ctx* ctx, const double* d_etb, const double* d_w, long long ndim, int ncol, const double* d_en,
               int nw, double sme, long long nkpt, double* d_out) {
  if (ncol < 1 || ncol > 4) return set_err(ctx, WTBG_ERR_ARG, "dos: 1 to 4 weight columns");
  k_dos<<<nw, 256, 0, ctx->stream>>>(d_etb, d_w, ndim, ncol, d_en, nw, sme, 1.0 / (double)nkpt, d_out);
  WTBG_COUNT(ctx, 1);
  CKL("k_dos");
  return 0;
}

// ---------------------------------------------------------------------------------------
// Allocation-free entry point.  The scratch of the three spectrum kernels (Re/Im sums per
// component and photon energy, and eta) lives in this fixed file-scope device array instead
// of context buffers, so the call performs no device allocation.  Host code must not use
// the symbol itself as an address: the device address belongs to the CUDA context that is
// current, so it is looked up with cudaGetSymbolAddress on every call made outside stream
// capture (a cheap query that allocates nothing) and remembered per context; a call made
// while its stream is being captured uses the remembered address of the current context.
namespace {
constexpr int kNoAllocMaxNw = 8192;
constexpr int kNoAllocMaxComp = 8;
constexpr size_t kNoAllocScratch = 2 * (size_t)kNoAllocMaxComp * kNoAllocMaxNw + 32;

typedef int (*CtxGetCurrentFn)(void**);   // cuCtxGetCurrent(CUcontext*)
std::mutex g_noalloc_mu;
std::map<void*, double*> g_noalloc_ptr;   // current CUDA context -> scratch address in it

int noalloc_fail(char* errbuf, int errlen, int code, const char* msg) {
  if (errbuf && errlen > 0) snprintf(errbuf, (size_t)errlen, "%s", msg);
  return code;
}

// the CUcontext current on this host thread (nullptr if the driver entry is unavailable)
void* current_context() {
  static CtxGetCurrentFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<CtxGetCurrentFn>(p);
  });
  void* c = nullptr;
  if (fn && fn(&c) != 0) c = nullptr;
  return c;
}
}  // namespace

static __device__ __align__(256) double g_spectrum_scratch[kNoAllocScratch];

extern "C" int wtbg_spectrum_noalloc(int n, int ncomp, const double* d_ebse, const double* d_fosc, const int* rtype,
                                     const int* ngrid, double vcell3d, double ebse0, double ebsef, double numbse,
                                     double sme, int renorm, double spinf, double* d_omega, float* d_eps,
                                     void* stream, char* errbuf, int errlen) {
  if (!d_ebse || !d_fosc || !rtype || !ngrid || !d_omega || !d_eps)
    return noalloc_fail(errbuf, errlen, WTBG_ERR_ARG, "spectrum_noalloc: null pointer");
  const int nw = (int)numbse;
  if (n <= 0 || nw < 2 || ncomp < 1)
    return noalloc_fail(errbuf, errlen, WTBG_ERR_ARG, "spectrum_noalloc: bad sizes");
  if (nw > kNoAllocMaxNw || ncomp > kNoAllocMaxComp)
    return noalloc_fail(errbuf, errlen, WTBG_ERR_UNSUPPORTED,
                        "spectrum_noalloc: NESPEC above 8192 or more than 8 components exceeds the fixed scratch");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return noalloc_fail(errbuf, errlen, WTBG_ERR_CUDA, "spectrum_noalloc: no current device");
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
    cudaGetLastError();
    return noalloc_fail(errbuf, errlen, WTBG_ERR_CUDA, "spectrum_noalloc: cannot query the stream");
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    void* cctx = current_context();
    if (cap == cudaStreamCaptureStatusNone) {
      // outside capture: resolve the address in the context that is current now (after a
      // cudaDeviceReset or under another context the old address would be invalid)
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_spectrum_scratch);
      if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return noalloc_fail(errbuf, errlen, WTBG_ERR_CUDA, "spectrum_noalloc: cudaGetSymbolAddress failed");
      }
      scratch = static_cast<double*>(p);
      if (cctx) g_noalloc_ptr[cctx] = scratch;
    } else {
      auto it = cctx ? g_noalloc_ptr.find(cctx) : g_noalloc_ptr.end();
      if (it == g_noalloc_ptr.end())
        return noalloc_fail(errbuf, errlen, WTBG_ERR_STATE,
                            "spectrum_noalloc: first call in this CUDA context made under stream capture; "
                            "call once before capturing");
      scratch = it->second;
    }
  }
  double* re = scratch;
  double* im = re + (size_t)ncomp * nw;
  double* eta = im + (size_t)ncomp * nw;
  SpecRtype rt{};
  for (int c = 0; c < ncomp; ++c) rt.rt[c] = rtype[c];
  const double baux = (double)(float)(ngrid[0] * ngrid[1] * ngrid[2]) * vcell3d;
  const double caux = (double)180.90f / (baux * 1.0);
  k_avgsme<<<1, 32, 0, s>>>(d_ebse, n, sme, eta);
  const int threads = 256;
  const int blocks = (nw * 32 + threads - 1) / threads;
  switch (ncomp) {
#define WTBG_SPEC_CASE(K)                                                                                    \
  case K:                                                                                                    \
    k_spectrum<K><<<blocks, threads, 0, s>>>(d_ebse, d_fosc, n, eta, ebse0, ebsef, numbse, nw, caux, rt,     \
                                             d_omega, re, im);                                               \
    break;
    WTBG_SPEC_CASE(1) WTBG_SPEC_CASE(2) WTBG_SPEC_CASE(3) WTBG_SPEC_CASE(4)
    WTBG_SPEC_CASE(5) WTBG_SPEC_CASE(6) WTBG_SPEC_CASE(7) WTBG_SPEC_CASE(8)
#undef WTBG_SPEC_CASE
    default: break;
  }
  k_renorm_out<<<1, 32, 0, s>>>(d_ebse, d_omega, re, im, nw, ncomp, renorm, spinf, d_eps);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(errbuf, errlen, WTBG_ERR_CUDA, cudaGetErrorString(e));
  return WTBG_OK;
}
