/*
 * wtbgpu.h -- C-ABI of libwtbgpu.so, the B200 (sm_100a) implementation of the
 * WanTiBEXOS Bethe-Salpeter exciton + optics path.
 *
 * The reference has no plugin or FFI layer: its boundary is the set of Fortran
 * subroutines that the driver (wtb_main.f90) calls.  Each entry point below
 * replaces one of those stages and is what a Fortran ISO_C_BINDING interface
 * (or the bundled C++ driver) binds.  Conventions:
 *   - arrays are column-major (Fortran order), caller-allocated host memory;
 *   - complex arrays are interleaved (re, im) doubles, i.e. complex(c_double_complex);
 *   - every call returns a status: 0 = OK, < 0 = error (see wtbg_error_string);
 *   - one context = one device + one CUDA stream, used from one host thread;
 *   - large arrays (H(k) eigenvectors, BSE matrix, reflectors) stay on the device.
 */
#ifndef WTBGPU_H
#define WTBGPU_H

#ifdef __cplusplus
extern "C" {
#endif

enum wtbg_status {
  WTBG_OK = 0,
  WTBG_ERR_ARG = -1,          /* invalid argument (size, pointer, option)                 */
  WTBG_ERR_CUDA = -2,         /* CUDA runtime error (message in wtbg_last_error)          */
  WTBG_ERR_OOM = -3,          /* device allocation failed                                  */
  WTBG_ERR_NOCONV = -4,       /* an iterative device solver hit its iteration cap          */
  WTBG_ERR_STATE = -5,        /* call order violated (e.g. solve before build)            */
  WTBG_ERR_BANDWINDOW = -6,   /* nv > nocp or nc > w - nocp at some k (quantumnumbers2)   */
  WTBG_ERR_NOEMPTY = -7,      /* no eigenvalue above E_F at some k (nocp undefined)       */
  WTBG_ERR_UNSUPPORTED = -8,  /* size or option outside what this build supports          */
  WTBG_ERR_NOCUDA = -9        /* no CUDA device available                                  */
};

/* Coulomb potential selector: the COULOMB_POT= deck values of matrizelbse
 * (subroutines/bse_subs.f90:49-93). */
enum wtbg_coulomb_type {
  WTBG_V2DK = 1, WTBG_V3D = 2, WTBG_V3DL = 3, WTBG_V2DT = 4, WTBG_V2DT2 = 5,
  WTBG_V2DOH = 6, WTBG_V2DRK = 7, WTBG_V1DT = 8, WTBG_V0DT = 9
};

/* Arguments of the coulomb_pot.f90 functions as matrizelbse passes them
 * (bse_subs.f90:2-93): KTOL, EDIEL_T/EDIEL/EDIEL_B, LC, EDIEL_Z, W_COUL, R_0, ngrid. */
typedef struct wtbg_coulomb {
  int coultype;       /* enum wtbg_coulomb_type */
  int ngrid[3];
  double ktol;
  double ediel[3];    /* ediel(1..3) = EDIEL_T, EDIEL, EDIEL_B */
  double lc, ez, w, r0;
} wtbg_coulomb;

typedef struct wtbg_ctx wtbg_ctx;

/* ---- context ------------------------------------------------------------ */
int wtbg_create(wtbg_ctx** ctx, int device);
int wtbg_destroy(wtbg_ctx* ctx);
const char* wtbg_error_string(int status);
const char* wtbg_last_error(const wtbg_ctx* ctx);
/* Milliseconds spent on the device by the last wtbg_* call on this context
 * (CUDA events on the context stream around that call's launches). */
double wtbg_last_device_ms(const wtbg_ctx* ctx);

/* Counters of the device work issued by this context since the last reset: kernel
 * launches, and (when profiling is on) CUDA-event time and algorithmic HBM bytes of the
 * two bandwidth-bound kernels of the path, the Hermitian matrix-vector product of the
 * tridiagonalisation and the BSE matrix build. */
typedef struct wtbg_stats {
  long long launches;
  long long hemv_launches;
  double hemv_ms;
  double hemv_bytes;
  long long build_launches;
  double build_ms;
  double build_bytes;
  long long fast_launches;   /* tensor-core products (k_fastprod), timed when profiling */
  double fast_ms;
  double fast_bytes;         /* algorithmic: 8 N^2 (bf16 hi/lo planes of Re H, Im H) per product */
  long long dav_fast_iters;  /* Davidson iterations on the tensor-core product (last call) */
  long long dav_fp64_iters;  /* Davidson iterations on the FP64 product (last call) */
  long long her2k_launches;  /* trailing rank-2k updates (k_her2k), timed when profiling */
  double her2k_ms;
  double her2k_flops;        /* algorithmic: 16 real flops x 2 x panel width per lower-triangle element */
  double tri_ms;             /* whole tridiagonalisation (profiling) */
  double tdsolve_ms;         /* tridiagonal eigenvalues + inverse iteration + oscillators (profiling) */
  long long dav_fallbacks;   /* wtbg_bse_lowest calls that fell back to the dense FP64 solve */
  double stage1_ms;          /* two-stage reduction: dense -> band (profiling) */
  double stage2_ms;          /* two-stage reduction: band -> tridiagonal (profiling) */
  double panel_ms;           /* two-stage: panel QR (profiling) */
  double hemm_ms;            /* two-stage: X = A22 V on the FP64 tensor cores (profiling) */
  double hemm_flops;         /* algorithmic: 8 m^2 nref per panel */
} wtbg_stats;
int wtbg_set_profiling(wtbg_ctx* ctx, int on);
int wtbg_get_stats(const wtbg_ctx* ctx, wtbg_stats* out);
int wtbg_reset_stats(wtbg_ctx* ctx);

/* Reduction used by the dense solves (wtbg_bse_solve, the Q eigenvalues): 0 = automatic (the
 * two-stage reduction, dense -> band of width 32 on the FP64 tensor cores -> tridiagonal by
 * bulge chasing, for N >= 2048 where its panels fit on the device; else one-stage),
 * 1 = one-stage (blocked Householder with a Hermitian mat-vec per column), 2 = two-stage
 * wherever it fits, 3 = as 2 with the bulge chasing run one warp per sweep instead of one CTA
 * of four warps per sweep (for comparison).  Both give the tridiagonal form of ZHETRD('L') up to rounding; the eigenvalues,
 * oscillator strengths and vectors agree within the tolerances of the dense path.  No counterpart
 * in the reference (its ZHEEV is MKL's). */
int wtbg_set_reduction(wtbg_ctx* ctx, int mode);

/* ---- model: replaces the module globals filled by hamiltonian_input_read
 *      (subroutines/module_input_read.f90:32-176).
 *      hre/him: hopmatrices/ihopmatrices (nvec,w,w); rvec (nvec,3); deg = ffactor(nvec);
 *      rlat (3,3) with rlat(i,:) = a_i; efermi; scs (scissors). */
int wtbg_set_model(wtbg_ctx* ctx, int w, int nvec, const double* hre, const double* him,
                   const int* rvec, const int* deg, const double* rlat,
                   double efermi, double scs);

/* ---- bands: replaces the per-k eigsys loop and band selection of bsesolver
 *      (bse_solver-tool-diel.f90:257-313; eigsys = hamiltonian_tb.f90:2-137).
 *      kpt (nk,3) Cartesian 1/Angstrom.  Outputs (each may be NULL):
 *      eigv (nk,nc+nv), vector (nk,nc+nv,w) complex (component 1 real, as ZHEEV('V','L')),
 *      nocpk (nk), egap (min direct gap).  The selected bands stay on the device. */
int wtbg_bands(wtbg_ctx* ctx, int nk, const double* kpt, int nv, int nc,
               double* eigv, double* vector, int* nocpk, double* egap);

/* ---- velocity: replaces the optsp loop (bse_solver-tool-diel.f90:365-396;
 *      optsp/hlm = optics.f90:1-156).  hr (N,5) complex: hrx, hry, hrz, hrsp, hrsm,
 *      N = nk*nc*nv in quantumnumbers2 order (k outer, c, v inner).  hr may be NULL. */
int wtbg_velocity(wtbg_ctx* ctx, double sme, double* hr);

/* ---- single-particle table: replaces vecres + Bubblem
 *      (bse_solver-tool-diel.f90:379-402, general_subs.f90:405-440).
 *      vecres (N,15) real(4), rows stably sorted by column 7. */
int wtbg_sp_table(wtbg_ctx* ctx, float* vecres);

/* ---- BSE kernel build: replaces the matrizelbse double loop
 *      (bse_solver-tool-diel.f90:431-458; bse_subs.f90:2-124; coulomb_pot.f90:2-432).
 *      The N x N matrix stays on the device (lower triangle, = conj of the reference's
 *      upper triangle). */
int wtbg_bse_build(wtbg_ctx* ctx, const wtbg_coulomb* p);

/* Copy the built matrix to the host with the reference's layout: hbse (N,N) complex,
 * upper triangle j >= i written, strictly lower part zero.  For checks on small N. */
int wtbg_bse_get_matrix(wtbg_ctx* ctx, double* hbse);

/* ---- dense solve + oscillators: replaces ZHEEV('V','U') and dielbsev/dielbsep
 *      (bse_solver-tool-diel.f90:485-602; bse_subs.f90:278-378).
 *      W (N) ascending; act (N,8) = xx, yy, zz, xy, xz, yz, sp, sm
 *      (xy/xz/yz zero unless dtfull, sp/sm zero unless cpol).  Requires wtbg_velocity. */
int wtbg_bse_solve(wtbg_ctx* ctx, int dtfull, int cpol, double* W, double* act);

/* Exciton eigenvectors n0..n1 (1-based, inclusive) after wtbg_bse_solve, for the
 * BSE_WF files (excwf2, bse_subs.f90:534-576).  A (N, n1-n0+1) complex, each vector
 * normalised with its last component real and >= 0. */
int wtbg_bse_eigvecs(wtbg_ctx* ctx, int n0, int n1, double* A);

/* ---- fast form: the nev lowest (largest = 0) or highest (largest = 1) eigenpairs of the
 *      built BSE matrix by block Davidson in FP64 (no counterpart in the reference: it
 *      replaces the dense ZHEEV when only the lowest excitons are needed; its oracle is the
 *      dense solve).  nb = block size (multiple of 8, nev <= nb <= 40); X0 (N,nb) complex
 *      optional initial block (NULL: unit vectors at the smallest / largest diagonal
 *      entries); convergence when every residual |H x - theta x| of the nev wanted states
 *      is below tol (eV) or after max_iter iterations.  Outputs W (nev), act (nev,8) as in
 *      wtbg_bse_solve (requires wtbg_velocity; may be NULL), X (N,nev) complex eigenvectors
 *      (may be NULL), iterations used and the largest final residual.  The BSE matrix is
 *      kept, so the call can be repeated (e.g. lowest and highest states). */
int wtbg_bse_davidson(wtbg_ctx* ctx, int nev, int nb, int largest, int max_iter, double tol,
                      const double* X0, int dtfull, int cpol, double* W, double* act, double* X,
                      int* iters, double* maxres);

/* ---- the nev lowest excitons with the dense fallback (no counterpart in the reference, whose
 *      only solver is ZHEEV; the fallback is that ZHEEV restated): block Davidson as
 *      wtbg_bse_davidson (largest = 0); when it ends with a residual at or above tol after
 *      max_iter iterations (or, with the temperature mode on and act requested, where the
 *      Davidson oscillators do not exist), the dense FP64 solve of wtbg_bse_solve runs on the
 *      same matrix and its nev lowest eigenpairs are returned, with *used_dense = 1 and the
 *      stats counter dav_fallbacks incremented.  W (nev), act (nev,8) as wtbg_bse_solve (may be
 *      NULL), X (N,nev) complex eigenvectors (may be NULL) normalised with the last component
 *      real and >= 0 in both cases; iters and maxres describe the Davidson run.  After a
 *      fallback the matrix has been overwritten by the reduction (as after wtbg_bse_solve) and
 *      wtbg_bse_eigvecs serves further vectors; without one the matrix is kept. */
int wtbg_bse_lowest(wtbg_ctx* ctx, int nev, int nb, int max_iter, double tol, const double* X0, int dtfull,
                    int cpol, double* W, double* act, double* X, int* iters, double* maxres, int* used_dense);

/* ---- bands of several models in one persistent launch (no counterpart in the reference,
 *      which loops eigsys per k per run): model m is the one set in ctxs[m] (all on one
 *      device; uneven w, nvec and meshes allowed) and gets exactly the state of
 *      wtbg_bands(ctxs[m], nk[m], kpt[m], nv[m], nc[m], ...): every (model, k) item runs in one
 *      kernel that takes items, largest w first, from a global counter.  kpt[m] (nk[m], 3)
 *      column-major; egap (nmod) or NULL.  Runs on ctxs[0]'s stream. */
int wtbg_bands_batch(wtbg_ctx* const* ctxs, int nmod, const int* nk, const double* const* kpt, const int* nv,
                     const int* nc, double* egap);

/* ---- eigsys for every band (hamiltonian_tb.f90:2-137 as the band-structure and DOS tools
 *      call it: bands-kpath-tool.f90:66-80, tdos-tool.f90:98-120): eig (nk, w) ascending with
 *      the scissors scs on the states above E_F, vec (nk, w, w) complex(8) = component m of
 *      band n at k (component 1 real, as ZHEEV('V','L')) or NULL, nocp (nk) or NULL.  Leaves
 *      the BSE state of the context alone. */
int wtbg_eigsys(wtbg_ctx* ctx, int nk, const double* kpt, double* eig, double* vec, int* nocp);

/* ---- DOS smearing of the DOS tool (endos, dos_subs.f90:102-152; gaussian,
 *      general_subs.f90:471-487): out(e, c) = (1/nkpt) sum_i weights(i, c) g(en(e) - etb(i)),
 *      g(x) = exp(-x^2 / (2 sme^2)) / (sme sqrt(2 pi)) with pi = acos(-1.) in real(4);
 *      weights (ndim, ncol) column-major, 1 <= ncol <= 4; out (nw, ncol). */
int wtbg_dos(wtbg_ctx* ctx, long long ndim, const double* etb, const double* weights, int ncol, long long nkpt,
             int nw, const double* en, double sme, double* out);

/* ---- temperature BSE (BSET=T / BSET_BND=T): with on = 1 every later call uses the
 *      occupation factor f_i = f_v - f_c (Fermi-Dirac, E_F = 0, kB = 8.617330350E-5 eV/K,
 *      T = 0 taken as 1E-8 K; fermidisteh, general_subs.f90:607-635) of each basis state:
 *      the kernel build scales the interaction part of the reference's upper-triangle row i
 *      by f_i (matrizelbsetemp, bse_subs_temp.f90:2-126; matrizelbsekqtemp :128-337), the
 *      sp table multiplies the strengths by f_i (bse_solver-tool-diel-temp.f90:416-423), and
 *      wtbg_bse_solve returns act = Re[(A^T h1) conj(A^T (h2 f))] (dielbseptemp,
 *      bse_subs_temp.f90:340-395).  The temperature gap correction (TA= VE/BE, gapcortemp /
 *      gapcortemp2) is a scissors shift the caller adds to scs in wtbg_set_model.  The fast
 *      form (wtbg_bse_spectrum_fast, oscillators of wtbg_bse_davidson) has no temperature
 *      form and returns WTBG_ERR_UNSUPPORTED while it is on. */
int wtbg_set_temperature(wtbg_ctx* ctx, int on, double temp);

/* ---- product used by the fast form (wtbg_bse_davidson, wtbg_bse_spectrum_fast, wtbg_bse_apply).
 *      mode 0: FP64 on CUDA cores (the lower triangle of H read once per product).
 *      mode 1: split-BF16 tensor-core product: the off-diagonal part of H is stored once per
 *      build as bf16 hi + lo planes of Re H and Im H (8 bytes per element, row-major), the
 *      vectors likewise, three bf16 products per pair accumulate in FP32, and the diagonal
 *      (band-energy differences) is applied in FP64; relative error ~1e-5 of |H_offdiag x|.
 *      No counterpart in the reference (its solver is ZHEEV on the full FP64 matrix). */
int wtbg_set_fast_product(wtbg_ctx* ctx, int mode);

/* ---- Y = H X for m vectors with the product selected by wtbg_set_fast_product; X, Y are
 *      complex(8) N x m column-major (interleaved re, im).  Requires wtbg_bse_build; keeps the
 *      matrix.  No counterpart in the reference. */
int wtbg_bse_apply(wtbg_ctx* ctx, int m, const double* X, double* Y);

/* ---- learned warm start for wtbg_bse_davidson (no counterpart in the reference).
 *      A per-transition MLP (3 layers, width 512, SiLU, BF16 weights with an FP32 master copy,
 *      FP32 accumulation on the tensor cores) maps band-edge data of each basis state
 *      (k, c, v) -- BSE diagonal, velocity matrix elements, k position, band indices -- and
 *      the sweep globals glob = {qx, qy, qz, r0, eps_env} to 5 complex coefficients per
 *      state; the 32-vector block is X[i,s] = sum_c coef * carrier_c[i] with carriers
 *      1, hx/|h|, hy/|h|, conj(hx)/|h|, conj(hy)/|h|.  Samples are the current basis of ctx
 *      (after wtbg_bands, wtbg_velocity and a build) plus the 32 lowest eigenvectors of the
 *      plain dense FP64 solve (A: N x 32 complex(8), column-major).  Training minimises the
 *      distance to the nearest orthonormal basis of span(A), min_R ||X - A R||^2 over unitary
 *      R (the polar factor of A^H X), per sample with Adam (hand-written forward, backward
 *      and update kernels).  The network is bound to ctx (device, stream). */
typedef struct wtbg_net wtbg_net;
int wtbg_net_create(wtbg_ctx* ctx, wtbg_net** net, unsigned long long seed);
int wtbg_net_destroy(wtbg_net* net);
long long wtbg_net_num_params(void);   /* flat fp32: W1[512][32] b1[512] W2[512][512] b2 W3[320][512] b3[320] */
int wtbg_net_get_params(wtbg_net* net, float* p);
int wtbg_net_set_params(wtbg_net* net, const float* p);
/* features F (N x 32 row-major, as rounded to bf16) and carriers CAR (5 x N complex(4)) of the
 * current basis; either may be NULL */
int wtbg_net_features(wtbg_net* net, const double* glob, float* F, float* CAR);
int wtbg_net_add_sample(wtbg_net* net, const double* glob, const double* A);
int wtbg_net_num_samples(wtbg_net* net);
/* epochs over samples [first, first+count) (count <= 0: all from first), mini-batches of
 * `batch` samples; loss_hist[epochs] gets the mean training loss per epoch (may be NULL) */
int wtbg_net_train(wtbg_net* net, int epochs, int batch, float lr, int first, int count, float* loss_hist);
int wtbg_net_eval_loss(wtbg_net* net, int first, int count, float* loss);
/* predicted block for the current basis of the bound context: X0 (N x 32 complex(8)) */
int wtbg_net_predict(wtbg_net* net, const double* glob, double* X0);
/* one forward + backward on explicit inputs (gradient check): F (nsamp*rows x 32, fp32),
 * CAR (5 x nsamp*rows complex(4)), A (32 x nsamp*rows complex(4), each sample's rows
 * orthonormal); loss and the flat gradient (layout of wtbg_net_get_params). rows % 8 == 0. */
int wtbg_net_loss_grad(wtbg_net* net, int nsamp, long long rows, const float* F, const float* CAR, const float* A,
                       float* loss, float* grad);
/* C (M x N, row-major, fp32) = A (M x K) B (N x K)^T with A, B rounded to bf16 and FP32
 * accumulation: the tcgen05 GEMM the network kernels use, exposed for checks. K % 8 == 0. */
int wtbg_gemm_bf16(wtbg_ctx* ctx, int M, int N, int K, const float* A, const float* B, float* C);

/* ---- fast form of the BSE spectrum: eps(omega) of bsedielraw (and bsedielrawpol) from the
 *      Haydock recursion on the built BSE matrix, nsteps Lanczos steps per chain closed by a
 *      square-root terminator (no counterpart in the reference; oracle = dense solve +
 *      optdiel).  Because the reference's oscillator has no conjugate on the exciton vector,
 *      sum_n f_n/(z - E_n) = u^H (z - H)^-1 u with u = conj(h).  The broadening follows
 *      avgsme: eta = sme + 10 (emax - e1) / N, with e1, emax the lowest and highest exciton
 *      energies (wtbg_bse_davidson gives both); imagrenorm uses e1.  eps (nw,2,8) as real(4):
 *      components xx, yy, zz, xy, xz, yz, sp, sm (xy/xz/yz only if dtfull, sp/sm only if cpol,
 *      else zero).  Requires wtbg_velocity and wtbg_bse_build; keeps the matrix. */
int wtbg_bse_spectrum_fast(wtbg_ctx* ctx, int nsteps, int dtfull, int cpol, double e1, double emax,
                           const int* ngrid, double vcell3d, double ebse0, double ebsef, double numbse,
                           double sme, int renorm, double spinf, double* omega, float* eps);

/* ---- spectrum: replaces the omega loop of bsedielraw with optdiel, avgsme and
 *      imagrenorm (bse_diel-tool.f90:137-210; optics.f90:160-390), and the same loop of
 *      bsedielrawpol, spdielraw and spdielrawpol (bse_diel-tool-pol.f90, sp_diel-tool.f90,
 *      sp_diel-tool-pol.f90).  ebse (n) and fosc (n,ncomp) are the values as read back from
 *      bse_opt_diel.dat / sp_optics.dat (and the -pol files); rtype (ncomp) is optdiel's
 *      rtype per column (1: Re eps includes the +1, 0: off-diagonal); vcell3d = |(a1 x a2).a3|.
 *      Outputs omega (nw) and eps (nw,2,ncomp) as real(4): eps(:,1,c) = real(spinf*Re),
 *      eps(:,2,c) = real(spinf*Im).  ncomp <= 8, nw = int(numbse). */
int wtbg_spectrum(wtbg_ctx* ctx, int n, int ncomp, const double* ebse, const double* fosc,
                  const int* rtype, const int* ngrid, double vcell3d, double ebse0,
                  double ebsef, double numbse, double sme, int renorm, double spinf,
                  double* omega, float* eps);

/* Allocation-free variant of wtbg_spectrum (no counterpart in the reference).
 * For hosts that cannot let a library allocate device memory: applications that hand out
 * all device memory from their own pool or a fixed arena, and services that must not call
 * cudaMalloc/cudaFree during a run because those calls can synchronise the whole device and
 * can fail with out-of-memory part-way through.  The caller owns every buffer:
 * d_ebse (n), d_fosc (n,ncomp), d_omega (nw) and d_eps (nw,2,ncomp) are DEVICE pointers on
 * the current device; rtype (ncomp) and ngrid (3) are host arrays; stream is a cudaStream_t
 * (NULL = default stream).  The kernels' scratch is a fixed static device array of
 * 2*8*8192+32 doubles (about 1 MB) that every GPU loading this library keeps until exit, so
 * nw = int(numbse) must be <= 8192 and ncomp <= 8; larger sizes return WTBG_ERR_UNSUPPORTED
 * with a message in errbuf.  The scratch address belongs to the CUDA context current on the
 * calling thread: every call made outside stream capture looks it up again
 * (cudaGetSymbolAddress, which allocates nothing), so calls after a cudaDeviceReset or under
 * a non-primary context are safe; a call made while `stream` is being captured reuses the
 * address found by an earlier call in the same context, so make one call in each context
 * before any stream capture (otherwise WTBG_ERR_STATE).  All calls share the
 * scratch: calls whose work overlaps on the GPU (different streams or host threads without
 * ordering) race.  Nothing in the scratch has to start at zero.  The call is asynchronous on
 * `stream`; no memory is allocated or freed. */
int wtbg_spectrum_noalloc(int n, int ncomp, const double* d_ebse, const double* d_fosc,
                          const int* rtype, const int* ngrid, double vcell3d, double ebse0,
                          double ebsef, double numbse, double sme, int renorm, double spinf,
                          double* d_omega, float* d_eps, void* stream, char* errbuf, int errlen);

/* ---- build the BSE matrix of one centre-of-mass momentum and keep it on the device
 *      (matrizelbsekq of bse_kpath-tool.f90:246-435 without the solve), for the fast form
 *      and the learned warm start at Q != 0.  Arguments as wtbg_bse_q_eigenvalues. */
int wtbg_bse_build_q(wtbg_ctx* ctx, int nk, const double* kptq, const double* q4, const wtbg_coulomb* p);

/* ---- exciton band structure: one centre-of-mass Q of bsebnds
 *      (bse_kpath-tool.f90:246-435; matrizelbsekq = bse_subs_kpath.f90:1-208).
 *      Uses the k-mesh bands of the last wtbg_bands call; kptq (nk,3) is the k+Q mesh
 *      of monhkhorst_packq (mhkpack_subs.f90:305-356) and q4 = (distance, qx, qy, qz)
 *      one row of the kpathbse path.  Builds the Q kernel with its exchange term and
 *      returns the eigenvalues W (N) ascending (ZHEEV('N','U')). */
int wtbg_bse_q_eigenvalues(wtbg_ctx* ctx, int nk, const double* kptq, const double* q4,
                           const wtbg_coulomb* p, double* W);

/* ---- Berry curvature (berryct2, berry_curvature_subs.f90:1-128, as berrycurv and
 *      berrycurvbz call it: berry_curvature_kpath-tool.f90, berry_curvature_bz-tool.f90):
 *      eigsys of every band at each k (scissors on the states above E_F), the velocity
 *      matrices dH/dk of hlm (optics.f90:1-97), and
 *        b_ab(k) = sum_{n <= nocp < i} -2 <n|h_a|i> conj(<n|h_b|i>) / ((E_n - E_i)^2 + gamma^2),
 *      pairs with |E_i - E_n| < degtol skipped.  The tools use gamma = 0.001 and degtol =
 *      0.0001, both single-precision literals (pass (double)0.001f, (double)0.0001f).
 *      kpt (nk,3); out (nk,6) = Im of b_xx, b_xy, b_xz, b_yy, b_yz, b_zz.  Leaves the BSE state
 *      of the context alone. */
int wtbg_berry(wtbg_ctx* ctx, int nk, const double* kpt, double gamma, double degtol, double* out);

/* ---- single-particle optical activity over the BZ (spoptpolbz, sp_opt_bz-tool.f90:81-175):
 *      eigsys of every band at each k, then over the band pairs of the BSE window
 *      (c = nocp_k+1 .. nocp_k+nc outer, v = nocp_k-nv+1 .. nocp of the FIRST k-point inner, the
 *      first nc*nv pairs) the sums of |h_a|^2 with h_a = <c|dH/dk_a|v> / (E_c - E_v + i sme),
 *      both terms of the denominator rounded to single precision as the reference's
 *      default-kind cmplx does.  out (nk,5) = x, y, z, sigma+, sigma- (sigma-pm with
 *      norm = f32(1/sqrt 2)).  WTBG_ERR_BANDWINDOW where a k-point has fewer than nc*nv pairs. */
int wtbg_sp_optbz(wtbg_ctx* ctx, int nk, const double* kpt, int nv, int nc, double sme, double* out);

/* ---- precision form (mode 1): the Fourier sums H(k) = sum_R e^{ik.R} H(R)/deg(R) of the band
 *      stage (hamiltonian_tb.f90:73-77) and the band overlaps <c|c'>, <v|v'> of the BSE kernel
 *      build (bse_subs.f90:2-124) run as 3-term split-BF16 GEMMs on the tensor cores with FP32
 *      accumulation; the per-k diagonalisation, the q -> 0 cell average, the velocities and the
 *      tridiagonalisation stay FP64.  mode 0 (default) is the FP64 form.  Switching the form
 *      discards the context's bands and matrix. */
int wtbg_set_precision(wtbg_ctx* ctx, int mode);

/* ---- exciton band structure, all Q of a path in one call (the Q loop of bsebnds,
 *      bse_kpath-tool.f90:246-435).  kptq holds nq blocks of (nk,3) k+Q meshes, q4 nq rows of
 *      (distance, qx, qy, qz); W (nq, N) receives each Q's eigenvalues ascending, identical to
 *      nq calls of wtbg_bse_q_eigenvalues.  With use_graph != 0 the tridiagonalisation (the
 *      launch-bound part: four launches per column) runs as one captured CUDA graph replayed
 *      for every Q after the first; the mat-vec chunk is autotuned per (device, N) on the
 *      first Q.  ms_q (nq, may be NULL) receives the device time of each Q. */
int wtbg_bse_q_batch(wtbg_ctx* ctx, int nk, int nq, const double* kptq, const double* q4,
                     const wtbg_coulomb* p, int use_graph, double* W, double* ms_q);

#ifdef __cplusplus
}
#endif
#endif /* WTBGPU_H */
