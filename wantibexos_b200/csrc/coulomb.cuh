// Screened Coulomb interactions W(k1 - k2) of subroutines/coulomb_pot.f90 as device
// functions (evaluated in the epilogue of the BSE kernel build, one value per (k, k')
// pair).  Every branch, threshold (|q| < KTOL) and float32 literal follows the reference:
//   cic = -(0.0904756)*10**3 and pi = acos(-1.) are real(4) values (coulomb_pot.f90:6-7),
//   alpha1 = 1.76 is real(4) (coulomb_pot.f90:8).
#pragma once
#include <cuda_runtime.h>

#include "../../include/wtbgpu.h"

struct CoulombDev {
  int type;
  double ktol;
  double vbz2d;     // 1/(nk * |a1 x a2|)
  double vbz3d;     // 1/(nk * |(a1 x a2).a3|)
  double cic;       // float32 -90.4756
  // V2DRK
  double eta, kappa, pb, pt, lc, w, r0;
  // V2DK
  double v2dk_r0, v2dk_ed, v2dk_q0;
  // V3DL
  double ed3;
  // V2DT
  double rc;
  // V0DT
  double cr;
  // V2DOH
  double ez;
  // V1DT
  double v1dt_q0;   // value at |q| -> 0 in both directions
};

// Bessel functions used by V1DT.  J0/J1 are CUDA's double-precision j0/j1; K0/K1 are
// evaluated from their integral representation K_nu(x) = int_0^inf exp(-x cosh t) cosh(nu t) dt
// (trapezoid rule, exponentially convergent) for x >= 0.1 and from the ascending series
// K0(x) = -(ln(x/2)+gamma) I0(x) + sum (x^2/4)^k/(k!)^2 H_k,
// K1(x) = 1/x + ln(x/2) I1(x) - x/4 sum (x^2/4)^k/(k!(k+1)!) (psi(k+1)+psi(k+2)) / 1 ... for small x.
__device__ inline double bessel_k_int(double x, int nu) {
  // trapezoid on t in [0, T]; integrand decays like exp(-x e^t / 2)
  double T = log(2.0 * (40.0 + fabs(log(x))) / x + 1.0) + 1.0;
  if (T < 1.0) T = 1.0;
  const int n = 400;
  const double h = T / n;
  double s = 0.5 * exp(-x);  // t = 0 (cosh(0)=1, cosh(nu*0)=1)
  for (int i = 1; i <= n; ++i) {
    const double t = i * h;
    const double f = exp(-x * cosh(t)) * (nu ? cosh(t) : 1.0);
    s += (i == n ? 0.5 : 1.0) * f;
  }
  return s * h;
}

__device__ inline double bessel_k_series(double x, int nu) {
  const double g = 0.57721566490153286061;
  const double y = 0.25 * x * x;
  if (nu == 0) {
    // K0 = -(ln(x/2) + gamma) I0(x) + sum_{k>=1} y^k/(k!)^2 H_k
    double term = 1.0, i0 = 1.0, s = 0.0, Hk = 0.0;
    for (int k = 1; k < 40; ++k) {
      term *= y / ((double)k * k);
      Hk += 1.0 / k;
      i0 += term;
      s += term * Hk;
    }
    return -(log(0.5 * x) + g) * i0 + s;
  }
  // K1 = 1/x + ln(x/2) I1(x) - (x/4) sum_{k>=0} y^k/(k!(k+1)!) (psi(k+1) + psi(k+2))
  double term = 1.0;  // y^k/(k!(k+1)!)
  double i1 = 0.0, s = 0.0;
  double psi1 = -g;   // psi(k+1)
  for (int k = 0; k < 40; ++k) {
    if (k > 0) {
      term *= y / ((double)k * (k + 1));
      psi1 += 1.0 / k;
    }
    const double psi2 = psi1 + 1.0 / (k + 1);
    i1 += term;
    s += term * (psi1 + psi2);
  }
  i1 *= 0.5 * x;
  return 1.0 / x + log(0.5 * x) * i1 - 0.25 * x * s;
}

__device__ inline double bessel_k(double x, int nu) {
  return (x < 0.1) ? bessel_k_series(x, nu) : bessel_k_int(x, nu);
}

// integralJ0pot (coulomb_pot.f90:437-469): 100-point trapezoid of r J0(r q) log r on
// r_i = (i-1)/(n-1)*rmax + 1e-4.
__device__ inline double integral_j0pot(double rmax, double q) {
  const int n = 100;
  const double eta = (double)1e-4f;   // "eta=1E-04" is a real(4) literal
  double res = 0.0;
  const double r1 = (0.0 / (n - 1.0)) * rmax + eta, r2 = (1.0 / (n - 1.0)) * rmax + eta;
  const double h = r2 - r1;
  double fprev = r1 * j0(r1 * q) * log(r1);
  for (int i = 2; i <= n; ++i) {
    const double r = ((i - 1.0) / (n - 1.0)) * rmax + eta;
    const double f = r * j0(r * q) * log(r);
    res = res + (h / 2.0) * (fprev + f);
    fprev = f;
  }
  return res;
}

__device__ inline double coulomb_eval(const CoulombDev& P, double dx, double dy, double dz) {
  const double modk = sqrt(dx * dx + dy * dy + dz * dz);
  switch (P.type) {
    case WTBG_V2DRK: {  // coulomb_pot.f90:276-340
      if (modk < P.ktol) return 0.0;
      const double aux1 = (1.0 - (P.pb * P.pt * exp(-2.0 * modk * P.eta * P.lc))) * P.kappa;
      const double aux2 = (1.0 - (P.pt * exp(-P.eta * modk * P.lc))) * (1.0 - (P.pb * exp(-P.eta * modk * P.lc)));
      const double aux3 = P.r0 * modk * exp(-modk * P.w);
      const double ew = (aux1 / aux2) + aux3;
      return (P.vbz2d * P.cic) * exp(-modk * P.w) * (1.0 / ew) * (1.0 / modk);
    }
    case WTBG_V2DK: {   // coulomb_pot.f90:2-51
      if (modk < P.ktol) return P.v2dk_q0;
      return P.vbz2d * (P.cic / P.v2dk_ed) * (1.0 / (modk * (1 + (P.v2dk_r0 * modk))));
    }
    case WTBG_V3D:      // coulomb_pot.f90:55-85
    case WTBG_V3DL: {   // coulomb_pot.f90:89-122
      if (modk < P.ktol) return 0.0;
      return P.vbz3d * (P.cic / P.ed3) * (1.0 / (modk * modk));
    }
    case WTBG_V2DT: {   // coulomb_pot.f90:126-183
      const double gz = fabs(dz);
      const double gpar = sqrt(dx * dx + dy * dy);
      const double rc = P.rc;
      if (gpar < P.ktol && gz < P.ktol) return (P.vbz3d * P.cic) * (-0.5 * rc * rc);
      if (gpar < P.ktol && gz >= P.ktol)
        return (P.vbz3d * P.cic) * (1.0 / (modk * modk)) * (1.0 - cos(gz * rc) - (gz * rc * sin(gz * rc)));
      const double aux1 = gz / gpar, aux2 = gpar * rc, aux3 = gz * rc;
      const double aux4 = aux1 * sin(aux3), aux5 = cos(aux3);
      return (P.vbz3d * P.cic) * (1.0 / (modk * modk)) * (1.0 + (exp(-aux2) * (aux4 - aux5)));
    }
    case WTBG_V0DT: {   // coulomb_pot.f90:187-228
      if (modk < P.ktol) return (P.vbz3d * P.cic) * (0.5) * P.cr * P.cr;
      return (P.vbz3d * P.cic) * (1.0 / (modk * modk)) * (1.0 - cos(P.cr * modk));
    }
    case WTBG_V2DT2: {  // coulomb_pot.f90:233-272
      if (modk < P.ktol) return 0.0;
      const double qxy = sqrt(dx * dx + dy * dy);
      return (P.vbz3d * P.cic) * (1.0 / (modk * modk)) * (1.0 - exp(-0.5 * qxy * P.lc) * cos(0.5 * P.lc * dz));
    }
    case WTBG_V2DOH: {  // coulomb_pot.f90:344-377
      if (modk < P.ktol) return 0.0;
      return (P.vbz2d * P.cic) * exp(-P.w * modk) * (1.0 / (P.ez * modk));
    }
    case WTBG_V1DT: {   // coulomb_pot.f90:381-432
      const double ax = fabs(dx);
      const double qyz = sqrt(dy * dy + dz * dz);
      if (ax < P.ktol && qyz >= P.ktol) return (P.vbz3d * P.cic) * integral_j0pot(P.lc, qyz);
      if (ax < P.ktol && qyz < P.ktol) return P.v1dt_q0;
      const double j0v = j0(qyz * P.lc), j1v = j1(qyz * P.lc);
      const double k0v = bessel_k(ax * P.lc, 0), k1v = bessel_k(ax * P.lc, 1);
      const double c1 = qyz * P.lc * j1v * k0v;
      const double c2 = ax * P.lc * j0v * k1v;
      return (P.vbz3d * P.cic) * (1.0 + c1 + c2);
    }
    default:
      return 0.0;
  }
}

// Host-side preparation of the parameter block (shared by the build kernels).
CoulombDev make_coulomb_dev(const wtbg_coulomb* p, const double* rlat_rowmajor);
