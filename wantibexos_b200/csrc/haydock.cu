// Haydock (Lanczos continued-fraction) spectrum of the BSE matrix: the fast form of the
// bsedielraw spectrum without any eigenvector (no reference counterpart; its oracle is the
// dense solve + optdiel).
//
// The reference's oscillator strength has no conjugate on the exciton vector,
// f_n = |sum_j A_jn h_j|^2 (bse_subs.f90:336-378), so with u = conj(h):
//   sum_n f_n / (z - E_n) = u^H (z - H)^-1 u,   z = omega + i*eta,
// and optdiel's sums (optics.f90:221-235) are Im: -Im G(z), Re: -Re G(z).  Lanczos on (H, u)
// gives G(z) = |u|^2 / (z - a_0 - b_0^2 / (z - a_1 - b_1^2 / ...)), closed with the
// square-root terminator of the asymptotic (a_inf, b_inf).  Off-diagonal tensor components
// use the polarisation identity Re(u_x^H R u_y) = (G_{x+y} - G_{x-y}) / 4.
#include <cmath>
#include <vector>

#include "common.cuh"

namespace {

constexpr int MAXC = 16;

// u_c = conj(combination of the h vectors) for each chain c
__global__ void k_chain_init(const double2* h, long long N, int ncomp, const int* code, double2* V) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= N) return;
  for (int c = 0; c < ncomp; ++c) {
    const int k = code[c];
    double2 u;
    if (k < 5) {
      u = h[(long long)k * N + i];
    } else {
      // 5: x+y 6: x-y 7: x+z 8: x-z 9: y+z 10: y-z
      const int a = (k <= 6) ? 0 : (k <= 8 ? 0 : 1);
      const int b = (k <= 6) ? 1 : 2;
      const double sg = (k % 2 == 1) ? 1.0 : -1.0;
      const double2 ha = h[(long long)a * N + i], hb = h[(long long)b * N + i];
      u = make_double2(ha.x + sg * hb.x, ha.y + sg * hb.y);
    }
    V[(long long)c * N + i] = cconj(u);
  }
}

// partial sums over row blocks for every chain: mode 0: |v|^2, mode 1: Re(v^H w)
__global__ void __launch_bounds__(256) k_chain_dot(const double2* Vv, const double2* Wv, long long N, int ncomp, int mode,
                                                   double* part) {
  __shared__ double red[8][MAXC];   // MAXC chains per block
  const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  const long long i = blockIdx.x * (long long)blockDim.x + tid;
  for (int c = 0; c < ncomp; ++c) {
    double s = 0.0;
    if (i < N) {
      const double2 v = Vv[(long long)c * N + i];
      if (mode == 0) s = v.x * v.x + v.y * v.y;
      else {
        const double2 w = Wv[(long long)c * N + i];
        s = v.x * w.x + v.y * w.y;
      }
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red[wp][c] = s;
  }
  __syncthreads();
  if (tid < ncomp) {
    double s = 0;
    for (int k = 0; k < 8; ++k) s += red[k][tid];
    part[(long long)blockIdx.x * MAXC + tid] = s;
  }
}

__global__ void k_chain_reduce(const double* part, int nparts, int ncomp, double* out) {
  const int c = threadIdx.x;
  if (c >= ncomp) return;
  double s = 0;
  for (int k = 0; k < nparts; ++k) s += part[(long long)k * MAXC + c];
  out[c] = s;
}

// w <- w - a v - b vp  (a = alpha_j, b = beta_{j-1})
__global__ void k_chain_axpy(double2* Wv, const double2* Vv, const double2* VPv, long long N, int ncomp, const double* a,
                             const double* b) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= N) return;
  for (int c = 0; c < ncomp; ++c) {
    const long long k = (long long)c * N + i;
    double2 w = Wv[k];
    const double2 v = Vv[k], vp = VPv[k];
    w.x -= a[c] * v.x + b[c] * vp.x;
    w.y -= a[c] * v.y + b[c] * vp.y;
    Wv[k] = w;
  }
}

// vp <- v, v <- w / sqrt(n2)
__global__ void k_chain_next(const double2* Wv, double2* Vv, double2* VPv, long long N, int ncomp, const double* n2) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= N) return;
  for (int c = 0; c < ncomp; ++c) {
    const long long k = (long long)c * N + i;
    VPv[k] = Vv[k];
    const double s = n2[c] > 0 ? 1.0 / sqrt(n2[c]) : 0.0;
    Vv[k] = cscale(Wv[k], s);
  }
}

__global__ void k_copy_scalar(const double* src, double* dst, int n, int sqrt_it) {
  const int c = threadIdx.x;
  if (c < n) dst[c] = sqrt_it ? sqrt(src[c]) : src[c];
}

// G(z) for every photon energy and chain; out re/im are -Re G and -Im G
__global__ void k_cfrac(const double* alpha, const double* beta, const double* norm2, int K, int ncomp, double ebse0,
                        double ebsef, double numbse, int nw, double eta, int terminate, double* om, double* gre,
                        double* gim) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nw * ncomp) return;
  const int j = t % nw, c = t / nw;
  const double w = ebse0 + (((ebsef - ebse0) * j) / (numbse - 1.));
  if (c == 0) om[j] = w;
  // complex arithmetic on (zr, zi)
  const double zr = w, zi = eta;
  double gr = 0.0, gi = 0.0;
  const double* a = alpha + (long long)c * K;
  const double* b = beta + (long long)c * K;
  if (terminate && K >= 8) {
    double ai = 0, bi = 0;
    for (int k = K / 2; k < K; ++k) {
      ai += a[k];
      bi += b[k];
    }
    ai /= (K - K / 2);
    bi /= (K - K / 2);
    // t = (z - a - sqrt((z-a)^2 - 4 b^2)) / (2 b^2), branch with Im t <= 0
    const double xr = zr - ai, xi = zi;
    const double dr = xr * xr - xi * xi - 4.0 * bi * bi, di = 2.0 * xr * xi;
    const double mod = sqrt(sqrt(dr * dr + di * di));
    const double ang = 0.5 * atan2(di, dr);
    double sr = mod * cos(ang), si = mod * sin(ang);
    if (si * zi < 0) {
      sr = -sr;
      si = -si;
    }
    const double den = 2.0 * bi * bi;
    if (den > 0) {
      gr = (xr - sr) / den;
      gi = (xi - si) / den;
    }
  }
  for (int k = K - 1; k >= 0; --k) {
    const double b2 = b[k] * b[k];
    const double dr = zr - a[k] - b2 * gr, di = zi - b2 * gi;
    const double dd = dr * dr + di * di;
    gr = dr / dd;
    gi = -di / dd;
  }
  const double n2 = norm2[c];
  gre[(long long)c * nw + j] = -n2 * gr;
  gim[(long long)c * nw + j] = -n2 * gi;
}

// eps from the chain Green functions: diagonal components directly, off-diagonal ones by
// polarisation; then imagrenorm against E_1 and real(spinf * x)
__global__ void k_haydock_eps(const double* om, const double* gre, const double* gim, int nw, int nout,
                              const int* ocode, double caux, double e1, int renorm, double spinf, double* re, double* im,
                              float* eps) {
  const int o = threadIdx.x;
  if (o >= nout) return;
  const int kind = ocode[2 * o], idx = ocode[2 * o + 1];
  double* ro = re + (long long)o * nw;
  double* io = im + (long long)o * nw;
  for (int j = 0; j < nw; ++j) {
    double r, i;
    if (kind == 0) {   // diagonal: chain idx
      r = gre[(long long)idx * nw + j];
      i = gim[(long long)idx * nw + j];
    } else {           // off-diagonal: chains idx (plus) and idx+1 (minus)
      r = 0.25 * (gre[(long long)idx * nw + j] - gre[(long long)(idx + 1) * nw + j]);
      i = 0.25 * (gim[(long long)idx * nw + j] - gim[(long long)(idx + 1) * nw + j]);
    }
    const double delta = (kind == 0) ? 1.0 : 0.0;
    ro[j] = delta + r * caux;
    io[j] = i * caux;
  }
  if (renorm) {
    const double aux = e1 - (double)0.15f;
    if (!(aux <= 0.000)) {
      int ibegin = 1;
      for (int i = 1; i <= nw; ++i) {
        if (om[i - 1] <= aux) ibegin = i;
        else break;
      }
      const double aux3 = (ibegin < nw) ? io[ibegin] : 0.0;
      for (int i = 1; i <= ibegin; ++i) io[i - 1] = 0.0;
      for (int i = ibegin + 1; i <= nw; ++i) {
        const double v = io[i - 1] - aux3;
        io[i - 1] = (v < 0.0) ? 0.0 : v;
      }
    }
  }
  for (int j = 0; j < nw; ++j) {
    eps[(long long)j + (long long)nw * (0 + 2 * o)] = (float)(spinf * ro[j]);
    eps[(long long)j + (long long)nw * (1 + 2 * o)] = (float)(spinf * io[j]);
  }
}

}  // namespace



// K Lanczos steps for every chain; alpha/beta (K x ncomp, chain-major) and |u|^2 to the host
int run_haydock(wtbg_ctx* ctx, int K, int ncomp, const int* codes, std::vector<double>& alpha, std::vector<double>& beta,
                std::vector<double>& norm2) {
  const long long N = ctx->N;
  if (ncomp < 1 || ncomp > MAXC) return set_err(ctx, WTBG_ERR_ARG, "haydock: 1..16 chains");
  cudaStream_t s = ctx->stream;
  const int m = ncomp <= 8 ? 8 : 16;   // block product width (chains padded with zero vectors)
  ENSURE(ctx->ws, (size_t)N * m * 16 * 3 + 4096);
  double2* V = ctx->ws.as<double2>();
  double2* VP = V + (size_t)N * m;
  double2* Wv = VP + (size_t)N * m;
  const int th = 256;
  const int nparts = (int)((N + th - 1) / th);
  ENSURE(ctx->tmp2, (size_t)nparts * MAXC * 8 + (size_t)(2 * K + 8) * MAXC * 8 + 1024);
  double* part = ctx->tmp2.as<double>();
  double* dal = part + (size_t)nparts * MAXC;            // [K][MAXC]
  double* dbe = dal + (size_t)K * MAXC;                   // [K][MAXC]
  double* dn2 = dbe + (size_t)K * MAXC;                   // [MAXC]
  double* db0 = dn2 + MAXC;                               // zeros (beta_{-1})
  ENSURE(ctx->istat, 64 * 4);
  int* dcode = ctx->istat.as<int>();
  CK(cudaMemcpyAsync(dcode, codes, ncomp * 4, cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(V, 0, (size_t)N * m * 16 * 3, s));
  CK(cudaMemsetAsync(db0, 0, MAXC * 8, s));
  k_chain_init<<<nparts, th, 0, s>>>(ctx->h.as<double2>(), N, ncomp, dcode, V); WTBG_COUNT(ctx, 1);
  k_chain_dot<<<nparts, th, 0, s>>>(V, V, N, ncomp, 0, part); WTBG_COUNT(ctx, 1);
  k_chain_reduce<<<1, 32, 0, s>>>(part, nparts, ncomp, dn2); WTBG_COUNT(ctx, 1);
  k_chain_next<<<nparts, th, 0, s>>>(V, V, VP, N, ncomp, dn2); WTBG_COUNT(ctx, 1);   // v = u/|u|, vp = u (reset below)
  CK(cudaMemsetAsync(VP, 0, (size_t)N * m * 16, s));
  CKL("haydock init");
  for (int j = 0; j < K; ++j) {
    if (int r = run_hemm_narrow(ctx, V, (int)N, m, Wv, (int)N)) return r;
    k_chain_dot<<<nparts, th, 0, s>>>(V, Wv, N, ncomp, 1, part); WTBG_COUNT(ctx, 1);
    k_chain_reduce<<<1, 32, 0, s>>>(part, nparts, ncomp, dal + (size_t)j * MAXC); WTBG_COUNT(ctx, 1);
    const double* bprev = (j == 0) ? db0 : dbe + (size_t)(j - 1) * MAXC;
    k_chain_axpy<<<nparts, th, 0, s>>>(Wv, V, VP, N, ncomp, dal + (size_t)j * MAXC, bprev); WTBG_COUNT(ctx, 1);
    k_chain_dot<<<nparts, th, 0, s>>>(Wv, Wv, N, ncomp, 0, part); WTBG_COUNT(ctx, 1);
    k_chain_reduce<<<1, 32, 0, s>>>(part, nparts, ncomp, dbe + (size_t)j * MAXC); WTBG_COUNT(ctx, 1);
    k_chain_next<<<nparts, th, 0, s>>>(Wv, V, VP, N, ncomp, dbe + (size_t)j * MAXC); WTBG_COUNT(ctx, 1);
    k_copy_scalar<<<1, 32, 0, s>>>(dbe + (size_t)j * MAXC, dbe + (size_t)j * MAXC, ncomp, 1); WTBG_COUNT(ctx, 1);
  }
  CKL("haydock steps");
  std::vector<double> ha((size_t)K * MAXC), hb((size_t)K * MAXC), hn(MAXC);
  CK(cudaMemcpyAsync(ha.data(), dal, ha.size() * 8, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(hb.data(), dbe, hb.size() * 8, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(hn.data(), dn2, MAXC * 8, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  alpha.assign((size_t)K * ncomp, 0.0);
  beta.assign((size_t)K * ncomp, 0.0);
  norm2.assign(ncomp, 0.0);
  for (int c = 0; c < ncomp; ++c) {
    norm2[c] = hn[c];
    for (int j = 0; j < K; ++j) {
      alpha[(size_t)c * K + j] = ha[(size_t)j * MAXC + c];
      beta[(size_t)c * K + j] = hb[(size_t)j * MAXC + c];
    }
  }
  return 0;
}

// eps(omega) from the Lanczos coefficients
int run_haydock_spectrum(wtbg_ctx* ctx, int K, int nchain, const double* alpha, const double* beta, const double* norm2,
                         int nout, const int* ocode, const int* ngrid, double vcell3d, double ebse0, double ebsef,
                         double numbse, double eta, double e1, int renorm, double spinf, double* d_om, float* d_eps) {
  const int nw = (int)numbse;
  cudaStream_t s = ctx->stream;
  ENSURE(ctx->sp_out, (size_t)(2 * nchain + 2 * nout) * nw * 8 + (size_t)(2 * K + 1) * nchain * 8 + 64 * 4 + 64);
  double* gre = ctx->sp_out.as<double>();
  double* gim = gre + (size_t)nchain * nw;
  double* re = gim + (size_t)nchain * nw;
  double* im = re + (size_t)nout * nw;
  double* da = im + (size_t)nout * nw;
  double* db = da + (size_t)K * nchain;
  double* dn = db + (size_t)K * nchain;
  int* doc = reinterpret_cast<int*>(dn + nchain);
  CK(cudaMemcpyAsync(da, alpha, (size_t)K * nchain * 8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(db, beta, (size_t)K * nchain * 8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dn, norm2, (size_t)nchain * 8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(doc, ocode, (size_t)nout * 2 * 4, cudaMemcpyHostToDevice, s));
  const int th = 128;
  k_cfrac<<<(nw * nchain + th - 1) / th, th, 0, s>>>(da, db, dn, K, nchain, ebse0, ebsef, numbse, nw, eta, 1, d_om, gre,
                                                    gim); WTBG_COUNT(ctx, 1);
  const double baux = (double)(float)(ngrid[0] * ngrid[1] * ngrid[2]) * vcell3d;
  const double caux = (double)180.90f / (baux * 1.0);
  k_haydock_eps<<<1, 32, 0, s>>>(d_om, gre, gim, nw, nout, doc, caux, e1, renorm, spinf, re, im, d_eps); WTBG_COUNT(ctx, 1);
  CKL("haydock spectrum");
  return 0;
}
