// ORACLE -- test infrastructure only.
//
// CPU FP64 restatement of the time step of the reference solver (Program
// Dubwise, jmsegret/IWrepo mode1_bbl).  It is the correctness reference for
// the B200 library and the timed CPU baseline; it is never linked into, or
// called by, the product library.  Only tests/, __graft_entry__.smoke() and
// the CPU-baseline legs of bench.py load it.
//
// The reference is Fortran 77 built with `ifort -autodouble -O3` (every REAL
// is 8 bytes; SSE2 code without FMA).  No Fortran compiler exists here, so the
// reference cannot be built; this file restates it routine by routine, with
// runtime dims instead of dim.h PARAMETERs, following the reference's
// evaluation order.  Build it with -ffp-contract=off (see oracle/Makefile).
// Each routine cites the reference lines it follows.
//
// Pins: tests/golden holds the reference's own numeric artefacts
// (testout.dat from testhelm, z_grid.dat, uveltest.dat / cfl.dat /
// minmaxtest.dat / avgint.dat of the shipped 2-D forced run) and
// tests/test_oracle_pins.py checks this file against them.

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/iw_b200.h"

namespace {

typedef std::complex<double> cd;

// ---------------------------------------------------------------------------
// Complex FFT (any correct FFT reproduces FFT99/CFFT99 to rounding; the
// reference's own algorithm, Temperton's, is not needed for semantics).
// ---------------------------------------------------------------------------
struct CFFT {
  int n = 0;
  std::vector<cd> W;  // W[e] = exp(-2 pi i e / n)
  void init(int n_) {
    n = n_;
    W.resize(n);
    for (int e = 0; e < n; ++e) {
      long double a = -2.0L * 3.14159265358979323846264338327950288L * e / n;
      W[e] = cd((double)std::cos(a), (double)std::sin(a));
    }
  }
  // out[k] = sum_j in[j*stride] * exp(sign 2 pi i jk/n); sign=-1 forward.
  void rec(int m, int istride, const cd* in, cd* out, int wstep, bool inv,
           cd* tmp) const {
    if (m == 1) {
      out[0] = in[0];
      return;
    }
    int r = (m % 4 == 0) ? 4 : (m % 2 == 0) ? 2 : (m % 3 == 0) ? 3 : (m % 5 == 0) ? 5 : m;
    int s = m / r;
    for (int q = 0; q < r; ++q) rec(s, istride * r, in + q * istride, out + q * s, wstep * r, inv, tmp);
    for (int i = 0; i < m; ++i) tmp[i] = out[i];
    for (int k = 0; k < s; ++k) {
      for (int p = 0; p < r; ++p) {
        int kk = k + s * p;
        cd acc(0.0, 0.0);
        for (int q = 0; q < r; ++q) {
          long e = ((long)q * kk) % m;
          cd w = W[(size_t)(e * wstep) % n];
          if (inv) w = std::conj(w);
          acc += tmp[q * s + k] * w;
        }
        out[kk] = acc;
      }
    }
  }
  void run(const cd* in, cd* out, bool inv) const {
    std::vector<cd> tmp(n);
    rec(n, 1, in, out, 1, inv, tmp.data());
  }
};

inline double sq(double x) { return x * x; }

// COMMON /penaltyparams/ and /comomega/ (comparampen.h).  The reference keeps
// them global; every column sets them before use, so one instance per column
// (per thread here) computes the same numbers.
struct Pen {
  std::vector<double> pa, pb, pg, pd, pt1, pt2;
  double omega = 0.0;
  explicit Pen(int ns = 0) : pa(ns, 0.0), pb(ns, 0.0), pg(ns, 0.0), pd(ns, 0.0), pt1(ns, 0.0), pt2(ns, 0.0) {}
};

struct Orc {
  iw_dims dm;
  iw_params pp;
  int nx, ny, nz, nzloc, nsubd, nzm, nxpp, nxh, nxhp, nyh, ndims;
  size_t ntot;
  double alpha, beta;  // 2 pi / xlen, 2 pi / ylen
  double scaley;
  // setup tables (comleng.h, comlegendre.h, comwave.h, comgridptxyz.h)
  std::vector<double> zpts, wg, alpol, dmat, d2mat, d3mat;  // alpol[j*nzloc+k]=P_j(z_k); dmat[k*nzloc+j]=D(k,j)
  std::vector<double> xw, yw, xsq, ysq, xg, yg, zg, zf;
  CFFT fx, fy;
  // state (comflow.h, commatrix.h, comrotpressbc.h)
  std::vector<double> F[4], Fn[4], Fnm[4];  // u,v,w,temp at n, n-1, n-2
  std::vector<double> S[4], Sn[4], Snm[4];  // NL terms
  std::vector<double> wnl, wviscrot;        // (nxpp,ny,2)
  std::vector<double> ub, vb, wb;           // calcuvwt's static locals
  double t = 0.0, dt;
  double fac1 = 1, fac2 = 0, fac3 = 0, bdf1 = 1, bdf2 = 0, bdf3 = 0, bdfv = 1;
  double facvel, fact;
  int istep = 0;
  // adaptive time step (COMMON /vardtflags/ ivardt, idtstep and cdt, comtime.h)
  double cdt = 1.0;
  int ivardt = 0, idtstep = 0;
  int istart = 0;  // main.f istart after a restart read (0: a new run)
  // animation dumps (solver.f:136-222): interval (0 = off), Tdump, counter
  double dtanim = 0, tdump = 0;
  int ianimc = 0;
  std::string anim_dir;
  int nlegspec = 0;  // ncalclegspec (0 = off)
  double tstart = 0;  // &mflags tstart (postp's time origin)
  std::string leg_dir;
  // penalty COMMON (comparampen.h) used by the single-call C API
  struct Pen* pen0 = nullptr;
  // filter tables
  std::vector<double> leg_sigma;  // specfilter(k) k=0..nzm
  // diagnostics of the last maxcalc / interface averaging
  double probe[2] = {0, 0};
  double mm[8], cfl[3];
  int cfl_idx[9];
  int mm_idx[8];
  int avg_count[4] = {0, 0, 0, 0};
  // oracle-fast factor cache: bit-identical to re-factoring every call
  bool cache_on = true;
  // Fourier filter as a plain scale instead of magnitude/phase (the two are
  // equal in exact arithmetic; acos/cos/sin adds noise of about
  // 1e-16*|fr|^2/|fi| when |fi| << |fr|).  Off = the reference's form.
  bool fourier_scale = false;
  struct Fac {
    std::vector<double> ab;
    std::vector<int> ipiv;
    std::vector<double> pen;  // tau1(1), tau2(nsubd) for the RHS rows
  };
  std::map<std::string, std::shared_ptr<Fac>> cache;

  size_t idx(int i, int j, int k) const { return (size_t)i + (size_t)nxpp * ((size_t)j + (size_t)ny * (size_t)k); }
};

// ---------------------------------------------------------------------------
// setup.f
// ---------------------------------------------------------------------------

// setup.f:334-361 legen: Legendre polynomials and derivatives at xc.
void legen(std::vector<double>& al, std::vector<double>& alp, int n, double xc) {
  al.assign(n + 2, 0.0);
  alp.assign(n + 2, 0.0);
  al[0] = 1.;
  al[1] = xc;
  alp[0] = 0;
  alp[1] = 1.;
  for (int k = 1; k <= n; ++k) {
    int kp = k + 1, km = k - 1;
    al[kp] = (2. * k + 1.) * xc * al[k] / kp - k * al[km] / kp;
  }
  for (int k = 1; k <= n; ++k) {
    int kp = k + 1, km = k - 1;
    alp[kp] = (2. * k + 1.) * (al[k] + xc * alp[k]) / kp - k * alp[km] / kp;
  }
}

// setup.f:486-518 jacobf (alp=bet=0: Legendre).
void jacobf(int n, double& poly, double& pder, double& polym1, double& pderm1, double& polym2,
            double& pderm2, double x) {
  const double alp = 0.0, bet = 0.0, rv = 1.0 + alp;
  double apb = alp + bet;
  poly = 1.0;
  pder = 0.0;
  if (n == 0) return;
  double polylst = poly, pderlst = pder;
  poly = rv * x;
  pder = rv;
  if (n == 1) return;
  double psave = 0, pdsave = 0;
  for (int k = 2; k <= n; ++k) {
    double a1 = 2. * k * (k + apb) * (2. * k + apb - 2.);
    double a2 = (2. * k + apb - 1.) * (alp * alp - bet * bet);
    double b3 = (2. * k + apb - 2.);
    double a3 = b3 * (b3 + 1.) * (b3 + 2.);
    double a4 = 2. * (k + alp - 1.) * (k + bet - 1.) * (2. * k + apb);
    double polyn = ((a2 + a3 * x) * poly - a4 * polylst) / a1;
    double pdern = ((a2 + a3 * x) * pder - a4 * pderlst + a3 * poly) / a1;
    psave = polylst;
    pdsave = pderlst;
    polylst = poly;
    poly = polyn;
    pderlst = pder;
    pder = pdern;
  }
  polym1 = polylst;
  pderm1 = pderlst;
  polym2 = psave;
  pderm2 = pdsave;
}

// setup.f:395-479 jacobl: Gauss-Lobatto-Legendre points, ascending.
void jacobl(int n, std::vector<double>& xcol) {
  const int kstop = 10;
  const double eps = 1.0e-12;
  std::vector<double> xjac(n + 3, 0.0);  // 1-based
  int np = n + 1;
  double pnp1p, pdnp1p, pnp, pdnp, pnm1p, pdnm1, pnp1m, pdnp1m, pnm, pdnm, pnm1m;
  jacobf(np, pnp1p, pdnp1p, pnp, pdnp, pnm1p, pdnm1, 1.0);
  jacobf(np, pnp1m, pdnp1m, pnm, pdnm, pnm1m, pdnm1, -1.0);
  double det = pnp * pnm1m - pnm * pnm1p;
  double rp = -pnp1p, rm = -pnp1m;
  double a = (rp * pnm1m - rm * pnm1p) / det;
  double b = (rm * pnp - rp * pnm) / det;
  xjac[1] = 1.0;
  int nh = (n + 1) / 2;
  double dth = 3.14159265 / (2 * n + 1);
  double cd_ = std::cos(2. * dth), sd = std::sin(2. * dth), cs = std::cos(dth), ss = std::sin(dth);
  for (int j = 2; j <= nh; ++j) {
    double x = cs;
    for (int k = 1; k <= kstop; ++k) {
      double pnp1, pdnp1, pn, pdn, pnm1;
      jacobf(np, pnp1, pdnp1, pn, pdn, pnm1, pdnm1, x);
      double poly = pnp1 + a * pn + b * pnm1;
      double pder = pdnp1 + a * pdn + b * pdnm1;
      double recsum = 0.0;
      for (int i = 1; i <= j - 1; ++i) recsum = recsum + 1.0 / (x - xjac[i]);
      double delx = -poly / (pder - recsum * poly);
      x = x + delx;
      if (std::fabs(delx) < eps) break;
    }
    xjac[j] = x;
    double cssave = cs * cd_ - ss * sd;
    ss = cs * sd + ss * cd_;
    cs = cssave;
  }
  xjac[np] = -1.0;
  int npp = n + 2;
  for (int i = 2; i <= nh; ++i) xjac[npp - i] = -xjac[i];
  if (n % 2 == 0) xjac[nh + 1] = 0.0;
  xcol.assign(n + 1, 0.0);
  for (int k = 0; k <= n; ++k) xcol[k] = xjac[n - k + 1];
}

// setup.f:527-600 quad (weights, Legendre table) and setup.f:636-798 derv
// (Costa-Don D, D2, D3 with negative-row-sum diagonals).
void setup_tables(Orc& o) {
  int n = o.nzm, N1 = o.nzloc;
  jacobl(n, o.zpts);
  o.wg.assign(N1, 0.0);
  o.alpol.assign((size_t)N1 * N1, 0.0);
  std::vector<double> al, alp;
  const double small = 1.0e-30;
  for (int k = 0; k <= n; ++k) {
    legen(al, alp, n, o.zpts[k]);
    o.wg[k] = 2. / ((double)(n * (n + 1)) * al[n] * al[n] + small);
    for (int j = 0; j <= n; ++j) o.alpol[(size_t)j * N1 + k] = al[j];
  }
  std::vector<double> c(N1);
  for (int k = 0; k <= n; ++k) {
    double prod = 1.;
    for (int l = 0; l <= n; ++l)
      if (l != k) prod = prod * (o.zpts[k] - o.zpts[l]);
    c[k] = prod;
  }
  auto& D = o.dmat;
  auto& D2 = o.d2mat;
  auto& D3 = o.d3mat;
  D.assign((size_t)N1 * N1, 0.0);
  D2 = D;
  D3 = D;
  const auto& x = o.zpts;
  for (int k = 0; k <= n; ++k)
    for (int j = 0; j <= n; ++j) D[k * N1 + j] = (k != j) ? c[k] / (c[j] * (x[k] - x[j])) : 0.;
  for (int k = 0; k <= n; ++k) {
    double sum = 0.;
    for (int j = 0; j <= n; ++j)
      if (k != j) sum = sum + D[k * N1 + j];
    D[k * N1 + k] = -sum;
  }
  for (int k = 0; k <= n; ++k)
    for (int j = 0; j <= n; ++j)
      D2[k * N1 + j] = (k != j) ? 2.0 * (D[k * N1 + k] * D[k * N1 + j] - D[k * N1 + j] / (x[k] - x[j])) : 0.;
  for (int k = 0; k <= n; ++k) {
    double sum = 0.;
    for (int j = 0; j <= n; ++j)
      if (k != j) sum = sum + D2[k * N1 + j];
    D2[k * N1 + k] = -sum;
  }
  for (int k = 0; k <= n; ++k)
    for (int j = 0; j <= n; ++j)
      D3[k * N1 + j] = (k != j) ? 3.0 * (D2[k * N1 + k] * D[k * N1 + j] - D2[k * N1 + j] / (x[k] - x[j])) : 0.;
  for (int k = 0; k <= n; ++k) {
    double sum = 0.;
    for (int j = 0; j <= n; ++j)
      if (k != j) sum = sum + D3[k * N1 + j];
    D3[k * N1 + k] = -sum;
  }
}

// filtering.f:1225-1243 specfilter
double specfilter(int k, int kc, int n, double p, double amp) {
  if (k >= kc) {
    double theta = (double)(k - kc) / (double)(n - kc);
    return std::exp(-amp * std::pow(theta, 2. * p));
  }
  return 1.;
}

// filtering.f:1248-1268 specfilter_fourier2d with kc = 0 (the caller passes
// the integer PARAMETER kcf = 0, filtering.f:823,871).
double specfilter_fourier2d(double ak, double akmax, int kc, double p, double amp) {
  double akc = akmax * (double)kc;
  if (ak >= akc) {
    double theta = (ak - akc) / (akmax - akc);
    return std::exp(-amp * std::pow(theta, 2. * p));
  }
  return 1.;
}

// setup.f:6-166 (setup) minus the file I/O and unused tables.
void setup(Orc& o) {
  setup_tables(o);
  o.xw.assign(o.nxhp, 0.0);
  o.xsq = o.xw;
  for (int i = 0; i < o.nxhp; ++i) {
    o.xw[i] = i * o.alpha;
    o.xsq[i] = o.xw[i] * o.xw[i];
  }
  o.yw.assign(o.ny, 0.0);  // yw(1) stays 0 when ny = 1 (nyh = 0)
  o.ysq = o.yw;
  for (int j = 1; j <= o.nyh; ++j) {
    o.yw[j - 1] = (j - 1) * o.beta;
    o.yw[o.ny - j] = -j * o.beta;
  }
  for (int j = 0; j < o.ny; ++j) o.ysq[j] = o.yw[j] * o.yw[j];
  double pi2 = 8.0 * std::atan(1.0);
  double xl = pi2 / o.alpha, yl = pi2 / o.beta;
  o.xg.resize(o.nx);
  for (int i = 0; i < o.nx; ++i) o.xg[i] = i * xl / o.nx;
  o.yg.resize(o.ny);
  for (int j = 0; j < o.ny; ++j) o.yg[j] = j * yl / o.ny;
  o.zg.resize(o.nz);
  o.zf.assign((size_t)o.nsubd * (o.nzloc - 1) + 2, 0.0);  // zf(1..nz2) at 1-based index
  for (int ks = 0; ks < o.nsubd; ++ks)
    for (int kl = 0; kl < o.nzloc; ++kl) {
      double zloc = 0.5 * o.pp.zh[ks] * (o.zpts[kl] + 1.0);
      o.zg[ks * o.nzloc + kl] = o.pp.z0[ks] + zloc;
      int k2 = ks * (o.nzloc - 1) + kl + 1;
      o.zf[k2] = o.pp.z0[ks] + zloc;
    }
  o.fx.init(o.nx);
  if (o.ndims == 3) o.fy.init(o.ny);
  int kc = (int)(o.pp.fackc * o.nzm);
  o.leg_sigma.resize(o.nzloc);
  for (int k = 0; k <= o.nzm; ++k) o.leg_sigma[k] = specfilter(k, kc, o.nzm, o.pp.p, o.pp.amp);
}

// ---------------------------------------------------------------------------
// horfft.f:2-69 with FFT991 (fft.f:1361-1501) and CFFT99 (fft.f:1-406)
// semantics.  Forward: x real -> half complex (1/nx, B(0)=B(N/2)=0), then y
// complex unscaled on LOT = nxh columns (the x-Nyquist column is never
// y-transformed), then everything times 1/ny.  Inverse: y (nxh columns),
// then x (Im of DC and Nyquist ignored), padding zero-filled.
// ---------------------------------------------------------------------------
void horfft(Orc& o, double* b, int is, int nk) {
  const int nx = o.nx, ny = o.ny, nxpp = o.nxpp, nxh = o.nxh;
  const size_t nxppy = (size_t)nxpp * ny;
#pragma omp parallel
  {
    std::vector<cd> zin(std::max(nx, ny)), zout(std::max(nx, ny));
#pragma omp for schedule(static)
    for (int kz = 0; kz < nk; ++kz) {
      double* a = b + (size_t)kz * nxppy;
      if (is == -1) {
        for (int j = 0; j < ny; ++j) {
          double* row = a + (size_t)j * nxpp;
          for (int i = 0; i < nx; ++i) zin[i] = cd(row[i], 0.0);
          o.fx.run(zin.data(), zout.data(), false);
          double sc = 1.0 / (double)nx;
          for (int m = 0; m <= nx / 2; ++m) {
            row[2 * m] = zout[m].real() * sc;
            row[2 * m + 1] = zout[m].imag() * sc;
          }
          row[1] = 0.0;
          row[nx + 1] = 0.0;
        }
        if (o.ndims == 3) {
          for (int m = 0; m < nxh; ++m) {
            for (int j = 0; j < ny; ++j) zin[j] = cd(a[(size_t)j * nxpp + 2 * m], a[(size_t)j * nxpp + 2 * m + 1]);
            o.fy.run(zin.data(), zout.data(), false);
            for (int j = 0; j < ny; ++j) {
              a[(size_t)j * nxpp + 2 * m] = zout[j].real();
              a[(size_t)j * nxpp + 2 * m + 1] = zout[j].imag();
            }
          }
        }
        for (size_t i = 0; i < nxppy; ++i) a[i] = o.scaley * a[i];
      } else {
        if (o.ndims == 3) {
          for (int m = 0; m < nxh; ++m) {
            for (int j = 0; j < ny; ++j) zin[j] = cd(a[(size_t)j * nxpp + 2 * m], a[(size_t)j * nxpp + 2 * m + 1]);
            o.fy.run(zin.data(), zout.data(), true);
            for (int j = 0; j < ny; ++j) {
              a[(size_t)j * nxpp + 2 * m] = zout[j].real();
              a[(size_t)j * nxpp + 2 * m + 1] = zout[j].imag();
            }
          }
        }
        for (int j = 0; j < ny; ++j) {
          double* row = a + (size_t)j * nxpp;
          zin[0] = cd(row[0], 0.0);
          zin[nx / 2] = cd(row[nx], 0.0);
          for (int m = 1; m < nx / 2; ++m) {
            zin[m] = cd(row[2 * m], row[2 * m + 1]);
            zin[nx - m] = std::conj(zin[m]);
          }
          o.fx.run(zin.data(), zout.data(), true);
          for (int i = 0; i < nx; ++i) row[i] = zout[i].real();
          row[nx] = 0.0;
          row[nx + 1] = 0.0;
        }
      }
    }
  }
}

// derv.f:212-275 dpdz: b(:,:,ks) = (2/zh(ks)) * D * a(:,:,ks).
void dpdz(const Orc& o, const double* a, double* b) {
  const int nzloc = o.nzloc;
  const size_t plane = (size_t)o.nxpp * o.ny;
#pragma omp parallel for schedule(static)
  for (int kk1 = 0; kk1 < o.nz; ++kk1) {
    int ks = kk1 / nzloc, k1 = kk1 % nzloc;
    double fac = 2. / o.pp.zh[ks];
    std::vector<double> sum(plane, 0.0);
    for (int k2 = 0; k2 < nzloc; ++k2) {
      int kk2 = ks * nzloc + k2;
      double dk = o.dmat[k1 * nzloc + k2];
      const double* src = a + (size_t)kk2 * plane;
      for (size_t p = 0; p < plane; ++p) sum[p] = sum[p] + dk * src[p];
    }
    double* dst = b + (size_t)kk1 * plane;
    for (size_t p = 0; p < plane; ++p) dst[p] = sum[p] * fac;
  }
}

// derv.f:279-329 dpdzcol over the whole subdomain column (nzbot=1, nztop=nzloc).
void dpdzcol(const Orc& o, const double* a, double* b, double ybar) {
  const int N = o.nzloc;
  for (int k1 = 0; k1 < N; ++k1) {
    double sum = 0.0;
    for (int k2 = 0; k2 < N; ++k2) sum = sum + o.dmat[k1 * N + k2] * a[k2];
    b[k1] = sum * (2. / ybar);
  }
}

// filtering.f:729-808 filter_legenpen.
void filter_legenpen(const Orc& o, const double* fin, double* fout) {
  const int N = o.nzloc, nzm = o.nzm;
  double a[IW_MAX_NZLOC], af[IW_MAX_NZLOC];
  for (int k = 0; k <= nzm; ++k) {
    double sum = 0.;
    for (int k1 = 0; k1 < N; ++k1) sum = sum + o.wg[k1] * fin[k1] * o.alpol[(size_t)k * N + k1];
    a[k] = (k == nzm) ? 0.5 * nzm * sum : (k + 0.5) * sum;
  }
  for (int k = 0; k <= nzm; ++k) af[k] = a[k] * o.leg_sigma[k];
  for (int k1 = 0; k1 < N; ++k1) {
    double sum = 0.;
    for (int k = 0; k <= nzm; ++k) sum = sum + af[k] * o.alpol[(size_t)k * N + k1];
    fout[k1] = sum;
  }
}

// filtering.f:811-983 filter_3dlegenfourier (magnitude/phase Fourier filter,
// then the Legendre filter of the real and imaginary parts, per subdomain).
void filter_3dlegenfourier(const Orc& o, double* f, int ifourier, int ilegen) {
  const int N = o.nzloc, nzm = o.nzm;
  double akmax = std::sqrt(o.xsq[o.nxhp - 1] + o.ysq[o.nyh]);
#pragma omp parallel for schedule(static)
  for (int j = 0; j < o.ny; ++j) {
    for (int ii = 0; ii < o.nxhp; ++ii) {
      int i = 2 * ii;
      double ak = std::sqrt(o.xsq[ii] + o.ysq[j]);
      for (int ks = 0; ks < o.nsubd; ++ks) {
        if (ifourier == 1) {
          for (int kl = 0; kl < N; ++kl) {
            int k = ks * N + kl;
            double fr = f[o.idx(i, j, k)], fi = f[o.idx(i + 1, j, k)];
            double fmag = std::sqrt(fr * fr + fi * fi);
            double cosc = fr / fmag, sinc = fi / fmag;
            if (o.fourier_scale) {
              double cf = specfilter_fourier2d(ak, akmax, 0, o.pp.pf, o.pp.amp);
              fr = fr * cf;
              fi = fi * cf;
            } else if (fmag != 0.) {
              double phase = 0.0;
              if (sinc >= 0.) phase = std::acos(cosc);
              if (sinc < 0.) phase = -std::acos(cosc);
              double cf = specfilter_fourier2d(ak, akmax, 0, o.pp.pf, o.pp.amp);
              double fmagf = fmag * cf;
              fr = fmagf * std::cos(phase);
              fi = fmagf * std::sin(phase);
            } else {
              fr = 0.;
              fi = 0.;
            }
            f[o.idx(i, j, k)] = fr;
            f[o.idx(i + 1, j, k)] = fi;
          }
        }
        if (ilegen == 1) {
          double ar[IW_MAX_NZLOC], ai[IW_MAX_NZLOC];
          for (int k = 0; k <= nzm; ++k) {
            double sumr = 0., sumi = 0.;
            for (int k1 = 0; k1 < N; ++k1) {
              int kg = ks * N + k1;
              double finr = f[o.idx(i, j, kg)], fini = f[o.idx(i + 1, j, kg)];
              sumr = sumr + o.wg[k1] * finr * o.alpol[(size_t)k * N + k1];
              sumi = sumi + o.wg[k1] * fini * o.alpol[(size_t)k * N + k1];
            }
            if (k == nzm) {
              ar[k] = 0.5 * nzm * sumr;
              ai[k] = 0.5 * nzm * sumi;
            } else {
              ar[k] = (k + 0.5) * sumr;
              ai[k] = (k + 0.5) * sumi;
            }
          }
          for (int k = 0; k <= nzm; ++k) {
            ar[k] = ar[k] * o.leg_sigma[k];
            ai[k] = ai[k] * o.leg_sigma[k];
          }
          for (int k1 = 0; k1 < N; ++k1) {
            int kg = ks * N + k1;
            double sumr = 0., sumi = 0.;
            for (int k = 0; k <= nzm; ++k) {
              sumr = sumr + ar[k] * o.alpol[(size_t)k * N + k1];
              sumi = sumi + ai[k] * o.alpol[(size_t)k * N + k1];
            }
            f[o.idx(i, j, kg)] = sumr;
            f[o.idx(i + 1, j, kg)] = sumi;
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// forcing.f helpers (mean stratification folded to constants)
// ---------------------------------------------------------------------------
double bruntz(const Orc& o) { return o.pp.brunt; }                            // forcing.f:156-162
double rhograd(const Orc& o) { return -(o.pp.rho0 * (sq(bruntz(o))) / o.pp.grav); }  // forcing.f:115-120
double rhomean(const Orc& o, double z) { return 1. + rhograd(o) * z; }      // forcing.f:134-141
double fzgaus(double z, double zcen, double zdim, double xbcrit) {           // forcing.f:264-280
  double r = (z - zcen) / zdim;
  return std::exp(-xbcrit * (r * r));
}
struct Wave {
  double pi2, xkcrit, xmcrit, xomega, twave, zdim;
};
Wave wave_params(const Orc& o) {  // main.f:328-348
  Wave w;
  w.pi2 = 8. * std::atan(1.0);
  w.zdim = o.pp.xlen;
  w.xkcrit = w.pi2 / o.pp.xlen;
  w.xmcrit = w.pi2 / (2. * o.pp.zlen);
  w.xomega = (bruntz(o) * w.xkcrit) / std::sqrt(w.xkcrit * w.xkcrit + w.xmcrit * w.xmcrit);
  w.twave = w.pi2 / w.xomega;
  return w;
}
double phit(double t, const Wave& w, double fwave) { return (t <= fwave * w.twave) ? 1. : 0.; }  // forcing.f:424-447

// ---------------------------------------------------------------------------
// solver.f:523-1206 rhsfm.  Inputs: u,v,w,temp and the 12 gradients in
// physical space; outputs su..st in spectral space; u,v,w,temp back to
// spectral space on return.
// ---------------------------------------------------------------------------
void rhsfm(Orc& o, std::vector<double>* G /*dudx,dudy,dudz,dvdx,...,dtdz*/) {
  const size_t ntot = o.ntot;
  double* u = o.F[0].data();
  double* v = o.F[1].data();
  double* w = o.F[2].data();
  double* tp = o.F[3].data();
  double* su = o.S[0].data();
  double* sv = o.S[1].data();
  double* sw = o.S[2].data();
  double* st = o.S[3].data();
  const double *dudx = G[0].data(), *dudy = G[1].data(), *dudz = G[2].data();
  const double *dvdx = G[3].data(), *dvdy = G[4].data(), *dvdz = G[5].data();
  const double *dwdx = G[6].data(), *dwdy = G[7].data(), *dwdz = G[8].data();
  std::vector<double> s1(ntot), s2(ntot), ox(ntot);
  const double omz = 0.0;  // main.f:440 omz = omega (an unset local: 0)
  for (size_t p = 0; p < ntot; ++p) s1[p] = -0.5 * u[p] * w[p];
  dpdz(o, s1.data(), su);
  for (size_t p = 0; p < ntot; ++p) s1[p] = -0.5 * v[p] * w[p];
  dpdz(o, s1.data(), sv);
  for (size_t p = 0; p < ntot; ++p) s1[p] = -0.5 * w[p] * w[p];
  dpdz(o, s1.data(), sw);
  const double coef = (sq(bruntz(o))) / rhograd(o);
  for (size_t p = 0; p < ntot; ++p) {
    su[p] = su[p] - 0.5 * (u[p] * dudx[p] + v[p] * (dudy[p] - 4. * omz) + w[p] * dudz[p]);
    sv[p] = sv[p] - 0.5 * (u[p] * (dvdx[p] + 4. * omz) + v[p] * dvdy[p] + w[p] * dvdz[p]);
    sw[p] = sw[p] - 0.5 * (u[p] * dwdx[p] + v[p] * dwdy[p] + w[p] * dwdz[p]);
    sw[p] = sw[p] + coef * tp[p];
  }
  // upwind interface penalty on the NL terms (solver.f:700-839)
  const double omega = 2. / (double)((o.nzloc + 1) * (o.nzloc + 2));
  for (int i = 0; i < o.nxpp; ++i)
    for (int j = 0; j < o.ny; ++j)
      for (int ks = 0; ks < o.nsubd; ++ks) {
        double ybar = o.pp.zh[ks];
        int kb = ks * o.nzloc, kt = ks * o.nzloc + o.nzloc - 1;
        double wbv = w[o.idx(i, j, kb)] + 0.0, wtv = w[o.idx(i, j, kt)] + 0.0;
        if (kb == 0) wbv = 0.;
        if (kt == o.nz - 1) wtv = 0.;
        double alpha0, tau1, gamma0, tau2;
        if (wbv > 0.) {
          alpha0 = wbv;
          tau1 = 0.5 / omega * (2. / ybar);
        } else {
          alpha0 = 0.;
          tau1 = 0.;
        }
        if (wtv < 0.) {
          gamma0 = std::fabs(wtv);
          tau2 = 0.5 / omega * (2. / ybar);
        } else {
          gamma0 = 0.;
          tau2 = 0.;
        }
        double* fields[4] = {u, v, w, tp};
        double* outs[4] = {su, sv, sw, st};
        for (int q = 0; q < 4; ++q) {
          double* f = fields[q];
          double* s = outs[q];
          double pcb = (kb == 0) ? 0. : alpha0 * f[o.idx(i, j, kb - 1)];
          s[o.idx(i, j, kb)] = s[o.idx(i, j, kb)] - tau1 * (alpha0 * f[o.idx(i, j, kb)] - pcb);
          double pct = (kt == o.nz - 1) ? 0. : gamma0 * f[o.idx(i, j, kt + 1)];
          s[o.idx(i, j, kt)] = s[o.idx(i, j, kt)] - tau2 * (gamma0 * f[o.idx(i, j, kt)] - pct);
        }
      }
  // background-wave terms are zero arrays (wavesetup not called), fcshear=0,
  // d2rhomeandz2=0: no-ops.  Virtual paddle (solver.f:942-960).  The loop of
  // solver.f:848 runs over k = 1..nz; its comment says the bottom point is
  // left out, and the reference's recorded run (uveltest.dat rows 641-1040,
  // the log `output`) was made that way: IW_PADDLE_ABOVE_BOTTOM starts at k = 2.
  if (o.pp.forcing) {
    Wave wv = wave_params(o);
    double ph = phit(o.t, wv, o.pp.fwave);
    double xa = o.pp.xacrit, um = o.pp.umax;
    for (int k = (o.pp.forcing == IW_PADDLE_ABOVE_BOTTOM ? 1 : 0); k < o.nz; ++k) {
      double zz = o.zg[k];
      double wzp = wv.xmcrit * std::cos(wv.xmcrit * zz);
      double wz = std::sin(wv.xmcrit * zz);
      for (int j = 0; j < o.ny; ++j)
        for (int i = 0; i < o.nx; ++i) {  // padding entries are ignored by the forward FFT
          double xx = o.xg[i];
          double arg = wv.xkcrit * xx - wv.xomega * o.t;
          double sinf = std::sin(arg), cosf = std::cos(arg);
          double fu = -((((((1 / wv.xkcrit) * (xa * um)) * wzp) * sinf) * um) / wv.zdim * ph);
          double fw = ((((xa * um) * wz) * cosf) * (um / wv.zdim)) * ph;
          double fr = ((xa * um) * wz * sinf) * -(1 / wv.xomega) * bruntz(o) * bruntz(o) * (o.pp.rho0 / o.pp.grav) *
                      (um / wv.zdim) * ph;
          su[o.idx(i, j, k)] = su[o.idx(i, j, k)] + fu;
          sw[o.idx(i, j, k)] = sw[o.idx(i, j, k)] + fw;
          st[o.idx(i, j, k)] = st[o.idx(i, j, k)] + fr;
        }
    }
  }
  // x and y derivative terms in spectral space (solver.f:1025-1105)
  auto addspec = [&](double* s, std::vector<double>& a1, std::vector<double>& a2) {
    for (int k = 0; k < o.nz; ++k)
      for (int j = 0; j < o.ny; ++j)
        for (int ii = 0; ii < o.nxhp; ++ii) {
          size_t pr = o.idx(2 * ii, j, k), pi = pr + 1;
          double X = o.xw[ii] * a1[pr] + o.yw[j] * a2[pr];
          double Y = o.xw[ii] * a1[pi] + o.yw[j] * a2[pi];
          s[pr] = s[pr] + (0. * X - 1. * Y);
          s[pi] = s[pi] + (0. * Y + 1. * X);
        }
  };
  for (size_t p = 0; p < ntot; ++p) {
    s1[p] = -0.5 * u[p] * u[p];
    s2[p] = -0.5 * u[p] * v[p];
  }
  horfft(o, su, -1, o.nz);
  horfft(o, s1.data(), -1, o.nz);
  horfft(o, s2.data(), -1, o.nz);
  addspec(su, s1, s2);
  for (size_t p = 0; p < ntot; ++p) {
    s1[p] = -0.5 * u[p] * v[p];
    s2[p] = -0.5 * v[p] * v[p];
  }
  horfft(o, sv, -1, o.nz);
  horfft(o, s1.data(), -1, o.nz);
  horfft(o, s2.data(), -1, o.nz);
  addspec(sv, s1, s2);
  for (size_t p = 0; p < ntot; ++p) {
    s1[p] = -0.5 * u[p] * w[p];
    s2[p] = -0.5 * v[p] * w[p];
  }
  horfft(o, sw, -1, o.nz);
  horfft(o, s1.data(), -1, o.nz);
  horfft(o, s2.data(), -1, o.nz);
  addspec(sw, s1, s2);
  // density perturbation (solver.f:1124-1198)
  for (size_t p = 0; p < ntot; ++p) s1[p] = -w[p] * tp[p];
  dpdz(o, s1.data(), ox.data());
  const double rg = rhograd(o);
  for (size_t p = 0; p < ntot; ++p) st[p] = st[p] + ox[p] - w[p] * rg;
  for (size_t p = 0; p < ntot; ++p) {
    s1[p] = -u[p] * tp[p];
    s2[p] = -v[p] * tp[p];
  }
  horfft(o, st, -1, o.nz);
  horfft(o, s1.data(), -1, o.nz);
  horfft(o, s2.data(), -1, o.nz);
  horfft(o, tp, -1, o.nz);
  addspec(st, s1, s2);
  horfft(o, u, -1, o.nz);
  horfft(o, v, -1, o.nz);
  horfft(o, w, -1, o.nz);
}

// solver.f:1210-1253 rotvisc: (kx^2+ky^2) w + i kx du/dz + i ky dv/dz at k0.
cd rotvisc(const Orc& o, const cd* us, const cd* vs, const cd* ws, double xw, double yw, double ybar, int k0) {
  const int N = o.nzloc;
  double fur[IW_MAX_NZLOC], fui[IW_MAX_NZLOC], fvr[IW_MAX_NZLOC], fvi[IW_MAX_NZLOC];
  double dfur[IW_MAX_NZLOC], dfui[IW_MAX_NZLOC], dfvr[IW_MAX_NZLOC], dfvi[IW_MAX_NZLOC];
  for (int k = 0; k < N; ++k) {
    fur[k] = us[k].real();
    fui[k] = us[k].imag();
    fvr[k] = vs[k].real();
    fvi[k] = vs[k].imag();
  }
  dpdzcol(o, fur, dfur, ybar);
  dpdzcol(o, fui, dfui, ybar);
  dpdzcol(o, fvr, dfvr, ybar);
  dpdzcol(o, fvi, dfvi, ybar);
  double xx = xw * xw, yy = yw * yw;
  double re = xx * ws[k0].real() + yy * ws[k0].real();
  double im = xx * ws[k0].imag() + yy * ws[k0].imag();
  re = re + (-xw * dfui[k0]);
  im = im + (xw * dfur[k0]);
  re = re + (-yw * dfvi[k0]);
  im = im + (yw * dfvr[k0]);
  return cd(re, im);
}

// solver.f:6-514 convec.
void convec(Orc& o) {
  const size_t ntot = o.ntot;
  double* w = o.F[2].data();
  for (int k = 0; k < o.nz; ++k) {
    w[o.idx(0, 0, k)] = 0.;
    w[o.idx(1, 0, k)] = 0.;
  }
  std::vector<double> G[12];
  for (auto& g : G) g.assign(ntot, 0.0);
  // z derivatives (dudz=G[2], dvdz=G[5], dwdz=G[8], dtdz=G[11])
  for (int q = 0; q < 4; ++q) dpdz(o, o.F[q].data(), G[3 * q + 2].data());
  for (int q = 0; q < 4; ++q) {
    const double* f = o.F[q].data();
    double* gx = G[3 * q].data();
    double* gy = G[3 * q + 1].data();
    for (int k = 0; k < o.nz; ++k)
      for (int j = 0; j < o.ny; ++j)
        for (int ii = 0; ii < o.nxhp; ++ii) {
          size_t pr = o.idx(2 * ii, j, k), pi = pr + 1;
          gx[pr] = -(o.xw[ii] * f[pi]);
          gx[pi] = o.xw[ii] * f[pr];
          gy[pr] = -(o.yw[j] * f[pi]);
          gy[pi] = o.yw[j] * f[pr];
        }
  }
  for (int q = 0; q < 4; ++q) horfft(o, o.F[q].data(), 1, o.nz);
  for (int g = 0; g < 12; ++g) horfft(o, G[g].data(), 1, o.nz);
  for (int q = 0; q < 4; ++q) std::fill(o.S[q].begin(), o.S[q].end(), 0.0);
  rhsfm(o, G);
  // wnl: extrapolated NL w-term at the walls (solver.f:267-284)
  for (int j = 0; j < o.ny; ++j)
    for (int i = 0; i < o.nxpp; ++i) {
      size_t b = o.idx(i, j, 0), tt = o.idx(i, j, o.nz - 1);
      o.wnl[(size_t)i + (size_t)o.nxpp * j] = o.fac1 * o.S[2][b] + o.fac2 * o.Sn[2][b] + o.fac3 * o.Snm[2][b];
      o.wnl[(size_t)i + (size_t)o.nxpp * (j + o.ny)] =
          o.fac1 * o.S[2][tt] + o.fac2 * o.Sn[2][tt] + o.fac3 * o.Snm[2][tt];
    }
  // keep the NL term at level n (uwork, solver.f:248-260)
  std::vector<double> snew[4];
  for (int q = 0; q < 4; ++q) snew[q] = o.S[q];
  for (int q = 0; q < 4; ++q)
    for (size_t p = 0; p < ntot; ++p) o.S[q][p] = o.fac1 * o.S[q][p] + o.fac2 * o.Sn[q][p] + o.fac3 * o.Snm[q][p];
  // rotational viscous term of the pressure BC (solver.f:318-394)
  const int N = o.nzloc;
  for (int j = 0; j < o.ny; ++j)
    for (int ii = 0; ii < o.nxhp; ++ii) {
      int i = 2 * ii;
      for (int side = 0; side < 2; ++side) {
        int ks = side == 0 ? 0 : o.nsubd - 1;
        int k0 = side == 0 ? 0 : N - 1;
        cd us[3][IW_MAX_NZLOC], vs[3][IW_MAX_NZLOC], ws[3][IW_MAX_NZLOC];
        const std::vector<double>* lv[3][3] = {{&o.F[0], &o.F[1], &o.F[2]},
                                               {&o.Fn[0], &o.Fn[1], &o.Fn[2]},
                                               {&o.Fnm[0], &o.Fnm[1], &o.Fnm[2]}};
        for (int l = 0; l < 3; ++l)
          for (int kl = 0; kl < N; ++kl) {
            int k = ks * N + kl;
            us[l][kl] = cd((*lv[l][0])[o.idx(i, j, k)], (*lv[l][0])[o.idx(i + 1, j, k)]);
            vs[l][kl] = cd((*lv[l][1])[o.idx(i, j, k)], (*lv[l][1])[o.idx(i + 1, j, k)]);
            ws[l][kl] = cd((*lv[l][2])[o.idx(i, j, k)], (*lv[l][2])[o.idx(i + 1, j, k)]);
          }
        double ybar = o.pp.zh[ks];
        cd r0 = rotvisc(o, us[0], vs[0], ws[0], o.xw[ii], o.yw[j], ybar, k0);
        cd r1 = rotvisc(o, us[1], vs[1], ws[1], o.xw[ii], o.yw[j], ybar, k0);
        cd r2 = rotvisc(o, us[2], vs[2], ws[2], o.xw[ii], o.yw[j], ybar, k0);
        double rr = o.fac1 * r0.real() + o.fac2 * r1.real() + o.fac3 * r2.real();
        double ri = o.fac1 * r0.imag() + o.fac2 * r1.imag() + o.fac3 * r2.imag();
        size_t base = (size_t)o.nxpp * (j + o.ny * side);
        o.wviscrot[base + i] = -(o.pp.xnu * rr);
        o.wviscrot[base + i + 1] = -(o.pp.xnu * ri);
      }
    }
  // u* by BDF (solver.f:402-430)
  std::vector<double> fold[4];
  for (int q = 0; q < 4; ++q) fold[q] = o.F[q];
  for (int q = 0; q < 4; ++q)
    for (size_t p = 0; p < ntot; ++p)
      o.F[q][p] = o.dt * o.S[q][p] + o.bdf1 * o.F[q][p] + o.bdf2 * o.Fn[q][p] + o.bdf3 * o.Fnm[q][p];
  // history rotation (solver.f:447-478)
  for (int q = 0; q < 4; ++q) {
    o.Snm[q].swap(o.Sn[q]);
    o.Sn[q] = snew[q];
    o.Fnm[q].swap(o.Fn[q]);
    o.Fn[q] = fold[q];
  }
  if (o.pp.ispecfilternl == 1)
    for (int q = 0; q < 4; ++q) filter_3dlegenfourier(o, o.F[q].data(), 1, 1);
}

// ---------------------------------------------------------------------------
// penalty.f, band_lu.f, bandludcmp.f, ludcmp.f
// ---------------------------------------------------------------------------
enum { IDIR = 0, INEU = 1, IROB = 2 };

// penalty.f:57-157 param_set.
void param_set(const Orc& o, const Pen& P, int ifbc, double& alpha0, double& beta0, double& tau0, double eps,
               double ybar) {
  const double omega = P.omega;
  if (ifbc == IDIR) {
    alpha0 = 1.;
    beta0 = 0.;
    double fac = o.pp.facdir * sq(2. / ybar);
    tau0 = fac * eps / (alpha0 * sq(omega));
  }
  if (ifbc == INEU) {
    alpha0 = 0.;
    beta0 = 1.;
    double fac = o.pp.facneumn * 2. / ybar;
    tau0 = fac / (beta0 * omega);
  }
  if (ifbc == IROB) {
    alpha0 = 1.;
    beta0 = 1.;
    double ck = alpha0 * omega / beta0;
    double dn = 1. / (omega * eps * beta0);
    double t1 = std::sqrt(sq(ck) + eps * ck);
    double t2 = 2. * ck - 2. * t1;
    double facm = ((1. / eps) >= 1.e5) ? o.pp.facrobin : 1.;
    double t3 = facm * dn * (eps + t2) * 2. / ybar;
    tau0 = t3;
  }
}

// penalty.f:9-53 penalty_setup (interior subdomains).
void penalty_setup(const Orc& o, Pen& P, double eps) {
  P.omega = 2. / (double)((o.nzloc + 1) * (o.nzloc + 2));
  for (int ks = 1; ks < o.nsubd - 1; ++ks) {
    double a0, b0, t0;
    param_set(o, P, IROB, a0, b0, t0, eps, o.pp.zh[ks]);
    P.pa[ks] = a0;
    P.pb[ks] = b0;
    P.pt1[ks] = t0;
    param_set(o, P, IROB, a0, b0, t0, eps, o.pp.zh[ks]);
    P.pg[ks] = a0;
    P.pd[ks] = b0;
    P.pt2[ks] = t0;
  }
}

// penalty.f:190-233: physical-boundary and end-interface parameters.
void penalty_ends(const Orc& o, Pen& P, double eps, int ifbcbot, int ifbctop) {
  const int ns = o.nsubd;
  double a0, b0, t0;
  param_set(o, P, ifbcbot, a0, b0, t0, eps, o.pp.zh[0]);
  P.pa[0] = a0;
  P.pb[0] = b0;
  P.pt1[0] = t0;
  if (ns > 1) {
    param_set(o, P, IROB, a0, b0, t0, eps, o.pp.zh[0]);
    P.pg[0] = a0;
    P.pd[0] = b0;
    P.pt2[0] = t0;
  }
  param_set(o, P, ifbctop, a0, b0, t0, eps, o.pp.zh[ns - 1]);
  P.pg[ns - 1] = a0;
  P.pd[ns - 1] = b0;
  P.pt2[ns - 1] = t0;
  if (ns > 1) {
    param_set(o, P, IROB, a0, b0, t0, eps, o.pp.zh[ns - 1]);
    P.pa[ns - 1] = a0;
    P.pb[ns - 1] = b0;
    P.pt1[ns - 1] = t0;
  }
}

// penalty.f:403-634 matrix_elmsetup (matrix part); a is nz x nz column major.
void matrix_assemble(const Orc& o, const Pen& P, double eps, std::vector<double>& a) {
  const int nz = o.nz, N = o.nzloc, ns = o.nsubd;
  a.assign((size_t)nz * nz, 0.0);
  auto A = [&](int r, int c) -> double& { return a[(size_t)r + (size_t)nz * c]; };  // 0-based
  const double* d = o.dmat.data();
  const double* d2 = o.d2mat.data();
  for (int ks = 0; ks < ns; ++ks) {
    double ybar = o.pp.zh[ks];
    double ybarl = ks > 0 ? o.pp.zh[ks - 1] : 0.0;
    double ybarr = ks < ns - 1 ? o.pp.zh[ks + 1] : 0.0;
    int km = ks * N;  // 0-based first row of the block is km
    for (int k1 = 0; k1 < N; ++k1)
      for (int k2 = 0; k2 < N; ++k2) A(km + k1, km + k2) = -(eps * sq(2. / ybar) * d2[k1 * N + k2]);
    for (int k1 = 0; k1 < N; ++k1) A(km + k1, km + k1) = A(km + k1, km + k1) + 1.;
    A(km, km) = A(km, km) + P.pt1[ks] * P.pa[ks];
    double cf = -(P.pt1[ks] * P.pb[ks] * eps * 2. / ybar);
    for (int k = 0; k < N; ++k) A(km, km + k) = A(km, km + k) + cf * d[0 * N + k];
    A(km + N - 1, km + N - 1) = A(km + N - 1, km + N - 1) + P.pt2[ks] * P.pg[ks];
    cf = +(P.pt2[ks] * P.pd[ks] * eps * 2. / ybar);
    for (int k = 0; k < N; ++k) A(km + N - 1, km + k) = A(km + N - 1, km + k) + cf * d[(N - 1) * N + k];
    if (ns > 1 && ks != 0) {
      A(km, km) = A(km, km) - 0.5 * P.pt1[ks] * P.pa[ks];
      cf = +(0.5 * P.pt1[ks] * P.pb[ks] * eps * 2. / ybar);
      for (int k = 0; k < N; ++k) A(km, km + k) = A(km, km + k) + cf * d[0 * N + k];
      for (int k = 0; k < N; ++k) A(km, km - N + k) = 0.;
      A(km, km - 1) = -(0.5 * P.pt1[ks] * P.pa[ks]);
      cf = +(0.5 * P.pt1[ks] * P.pb[ks] * eps * 2. / ybarl);
      for (int k = 0; k < N; ++k) A(km, km - N + k) = A(km, km - N + k) + cf * d[(N - 1) * N + k];
    }
    if (ns > 1 && ks != ns - 1) {
      A(km + N - 1, km + N - 1) = A(km + N - 1, km + N - 1) - 0.5 * P.pt2[ks] * P.pg[ks];
      cf = -(0.5 * P.pt2[ks] * P.pd[ks] * eps * 2. / ybar);
      for (int k = 0; k < N; ++k) A(km + N - 1, km + k) = A(km + N - 1, km + k) + cf * d[(N - 1) * N + k];
      for (int k = 0; k < N; ++k) A(km, km + N + k) = 0.;
      A(km + N - 1, km + N) = A(km + N - 1, km + N) - 0.5 * P.pt2[ks] * P.pg[ks];
      cf = -(0.5 * P.pt2[ks] * P.pd[ks] * eps * 2. / ybarr);
      for (int k = 0; k < N; ++k) A(km + N - 1, km + N + k) = A(km + N - 1, km + N + k) + cf * d[0 * N + k];
    }
  }
}

// bandludcmp.f:238-440 SGBTF2 (reached through SGBTRF with NB = 1, ILAENV
// ludcmp.f:7478-7492) with ISAMAX, SSWAP, SSCAL, SGER.  1-based AB(r,c).
int sgbtf2(int m, int n, int kl, int ku, double* ab, int ldab, int* ipiv) {
  auto AB = [&](int r, int c) -> double& { return ab[(size_t)(r - 1) + (size_t)ldab * (c - 1)]; };
  int kv = ku + kl, info = 0;
  for (int j = ku + 2; j <= std::min(kv, n); ++j)
    for (int i = kv - j + 2; i <= kl; ++i) AB(i, j) = 0.0;
  int ju = 1;
  for (int j = 1; j <= std::min(m, n); ++j) {
    if (j + kv <= n)
      for (int i = 1; i <= kl; ++i) AB(i, j + kv) = 0.0;
    int km = std::min(kl, m - j);
    // ISAMAX(km+1, AB(kv+1,j), 1)
    int jp = 1;
    double smax = std::fabs(AB(kv + 1, j));
    for (int i = 2; i <= km + 1; ++i) {
      if (std::fabs(AB(kv + i, j)) <= smax) continue;
      jp = i;
      smax = std::fabs(AB(kv + i, j));
    }
    ipiv[j - 1] = jp + j - 1;
    if (AB(kv + jp, j) != 0.0) {
      ju = std::max(ju, std::min(j + ku + jp - 1, n));
      if (jp != 1) {
        // SSWAP(ju-j+1, AB(kv+jp,j), ldab-1, AB(kv+1,j), ldab-1)
        for (int c = 0; c < ju - j + 1; ++c) std::swap(AB(kv + jp - c, j + c), AB(kv + 1 - c, j + c));
      }
      if (km > 0) {
        double r = 1.0 / AB(kv + 1, j);
        for (int i = 1; i <= km; ++i) AB(kv + 1 + i, j) = r * AB(kv + 1 + i, j);
        if (ju > j) {
          // SGER(km, ju-j, -1, AB(kv+2,j),1, AB(kv,j+1),ldab-1, AB(kv+1,j+1),ldab-1)
          for (int jj = 1; jj <= ju - j; ++jj) {
            double y = AB(kv + 1 - jj, j + jj);
            if (y != 0.0) {
              double temp = -1.0 * y;
              for (int ii = 1; ii <= km; ++ii)
                AB(kv + 1 + ii - jj, j + jj) = AB(kv + 1 + ii - jj, j + jj) + AB(kv + 1 + ii, j) * temp;
            }
          }
        }
      }
    } else if (info == 0) {
      info = j;
    }
  }
  return info;
}

// bandludcmp.f:883-1069 SGBTRS('N', nrhs=1) with SGER and STBSV
// (ludcmp.f:4698, upper, no transpose, non-unit).
void sgbtrs(int n, int kl, int ku, const double* ab, int ldab, const int* ipiv, double* b) {
  auto AB = [&](int r, int c) -> double { return ab[(size_t)(r - 1) + (size_t)ldab * (c - 1)]; };
  int kd = ku + kl + 1;
  if (kl > 0) {
    for (int j = 1; j <= n - 1; ++j) {
      int lm = std::min(kl, n - j);
      int l = ipiv[j - 1];
      if (l != j) std::swap(b[l - 1], b[j - 1]);
      double y = b[j - 1];
      if (y != 0.0) {
        double temp = -1.0 * y;
        for (int i = 1; i <= lm; ++i) b[j + i - 1] = b[j + i - 1] + AB(kd + i, j) * temp;
      }
    }
  }
  int k = kl + ku, kplus1 = k + 1;
  for (int j = n; j >= 1; --j) {
    if (b[j - 1] != 0.0) {
      int l = kplus1 - j;
      b[j - 1] = b[j - 1] / AB(kplus1, j);
      double temp = b[j - 1];
      for (int i = j - 1; i >= std::max(1, j - k); --i) b[i - 1] = b[i - 1] - temp * AB(l + i, j);
    }
  }
}

// band_lu.f:15-54 bandlu_solve: pack, factor, solve re and im.
int band_factor(const Orc& o, const std::vector<double>& a, std::vector<double>& ab, std::vector<int>& ipiv) {
  const int n = o.nz, kl = o.nzloc, ku = o.nzloc, ldab = 2 * kl + ku + 1;
  ab.assign((size_t)ldab * n, 0.0);
  ipiv.assign(n, 0);
  for (int j = 1; j <= n; ++j)
    for (int i = std::max(1, j - ku); i <= std::min(n, j + kl); ++i)
      ab[(size_t)(kl + ku + 1 + i - j - 1) + (size_t)ldab * (j - 1)] = a[(size_t)(i - 1) + (size_t)n * (j - 1)];
  return sgbtf2(n, n, kl, ku, ab.data(), ldab, ipiv.data());
}

struct BC {
  int ifbcbot, ifbctop;
  double bcrbot, bcibot, bcrtop, bcitop;
};

// penalty.f:162-251 penalty_main + helmv_penalty (255-397) + RHS part of
// matrix_elmsetup (588-605).  The factorisation is cached per (eps, BCs)
// when cache_on (identical to refactoring: the assembly is deterministic).
void penalty_main(Orc& o, Pen& P, double eps, const BC& bc, double* rhsinr, double* rhsini, double* fr, double* fi) {
  const int nz = o.nz, ns = o.nsubd;
  for (int k = 0; k < nz; ++k) {
    rhsinr[k] = -(rhsinr[k] * eps);
    rhsini[k] = -(rhsini[k] * eps);
  }
  penalty_ends(o, P, eps, bc.ifbcbot, bc.ifbctop);
  std::shared_ptr<Orc::Fac> fac;
  char key[128];
  snprintf(key, sizeof key, "%a|%d|%d|%a", eps, bc.ifbcbot, bc.ifbctop, P.pt1[0]);
  bool cacheable = o.cache_on;
#pragma omp critical(orc_cache)
  {
    if (cacheable) {
      auto it = o.cache.find(key);
      if (it != o.cache.end()) fac = it->second;
    }
  }
  if (!fac) {
    fac = std::make_shared<Orc::Fac>();
    std::vector<double> a;
    matrix_assemble(o, P, eps, a);
    band_factor(o, a, fac->ab, fac->ipiv);
    if (cacheable) {
#pragma omp critical(orc_cache)
      o.cache[key] = fac;
    }
  }
  for (int k = 0; k < nz; ++k) {
    fr[k] = rhsinr[k];
    fi[k] = rhsini[k];
  }
  if (bc.ifbcbot == IDIR) {
    fr[0] = rhsinr[0] + P.pt1[0] * bc.bcrbot;
    fi[0] = rhsini[0] + P.pt1[0] * bc.bcibot;
  } else {
    fr[0] = rhsinr[0] - P.pt1[0] * bc.bcrbot * eps;
    fi[0] = rhsini[0] - P.pt1[0] * bc.bcibot * eps;
  }
  if (bc.ifbctop == IDIR) {
    fr[nz - 1] = rhsinr[nz - 1] + P.pt2[ns - 1] * bc.bcrtop;
    fi[nz - 1] = rhsini[nz - 1] + P.pt2[ns - 1] * bc.bcitop;
  } else {
    fr[nz - 1] = rhsinr[nz - 1] + P.pt2[ns - 1] * bc.bcrtop * eps;
    fi[nz - 1] = rhsini[nz - 1] + P.pt2[ns - 1] * bc.bcitop * eps;
  }
  const int ldab = 3 * o.nzloc + 1;
  sgbtrs(nz, o.nzloc, o.nzloc, fac->ab.data(), ldab, fac->ipiv.data(), fr);
  sgbtrs(nz, o.nzloc, o.nzloc, fac->ab.data(), ldab, fac->ipiv.data(), fi);
}

// Legendre filter of a solution column per subdomain (calcuvwt.f:158-188).
void filter_column(const Orc& o, double* fr, double* fi) {
  const int N = o.nzloc;
  double tmp[IW_MAX_NZLOC];
  for (int ks = 0; ks < o.nsubd; ++ks) {
    filter_legenpen(o, fr + ks * N, tmp);
    std::memcpy(fr + ks * N, tmp, sizeof(double) * N);
    filter_legenpen(o, fi + ks * N, tmp);
    std::memcpy(fi + ks * N, tmp, sizeof(double) * N);
  }
}

// calcuvwt.f:2-746 / calcuvwt_noslip.f (BC variants) with update (826-901).
// Inputs: su..st = u*,v*,w*,temp* (spectral); outputs u,v,w,temp at n+1.
void calcuvwt(Orc& o, bool cpenspecfilter) {
  const int nz = o.nz, N = o.nzloc, ns = o.nsubd;
  const bool noslip = o.pp.bc_variant == IW_BC_NOSLIP;
  std::vector<double> phi(o.ntot, 0.0), dphidz(o.ntot, 0.0);
  const int ncol = o.nxhp * o.ny;
  // pressure (calcuvwt.f:87-222); phi(1,1,:) = 0
#pragma omp parallel for schedule(dynamic, 16)
  for (int c = 0; c < ncol; ++c) {
    int j = c / o.nxhp, ii = c % o.nxhp, i = 2 * ii;
    if (ii == 0 && j == 0) continue;
    Pen P(ns);
    double ak = o.xsq[ii] + o.ysq[j];
    double eps = 1. / ak;
    penalty_setup(o, P, eps);
    std::vector<double> rhsr(nz), rhsi(nz), fr(nz), fi(nz);
    double wr[IW_MAX_NZLOC], wi[IW_MAX_NZLOC], dwr[IW_MAX_NZLOC], dwi[IW_MAX_NZLOC];
    // divcolc (derv.f:35-85), divvel zeroed first
    for (int ks = 0; ks < ns; ++ks) {
      double ybar = o.pp.zh[ks];
      for (int kl = 0; kl < N; ++kl) {
        int k = ks * N + kl;
        wr[kl] = o.S[2][o.idx(i, j, k)];
        wi[kl] = o.S[2][o.idx(i + 1, j, k)];
      }
      dpdzcol(o, wr, dwr, ybar);
      dpdzcol(o, wi, dwi, ybar);
      for (int kl = 0; kl < N; ++kl) {
        int k = ks * N + kl;
        double ur = o.S[0][o.idx(i, j, k)], ui = o.S[0][o.idx(i + 1, j, k)];
        double vr = o.S[1][o.idx(i, j, k)], vi = o.S[1][o.idx(i + 1, j, k)];
        double dr = 0.0, di = 0.0;
        dr = dr + (0. * ur - o.xw[ii] * ui) + (0. * vr - o.yw[j] * vi);
        di = di + (0. * ui + o.xw[ii] * ur) + (0. * vi + o.yw[j] * vr);
        dr = dr + dwr[kl];
        di = di + dwi[kl];
        rhsr[k] = dr / o.dt;
        rhsi[k] = di / o.dt;
      }
    }
    BC bc;
    bc.ifbcbot = INEU;
    bc.ifbctop = INEU;
    size_t p1 = (size_t)i + (size_t)o.nxpp * j, p2 = (size_t)i + (size_t)o.nxpp * (j + o.ny);
    bc.bcrtop = o.wnl[p2] + o.wviscrot[p2];
    bc.bcrbot = o.wnl[p1] + o.wviscrot[p1];
    bc.bcitop = o.wnl[p2 + 1] + o.wviscrot[p2 + 1];
    bc.bcibot = o.wnl[p1 + 1] + o.wviscrot[p1 + 1];
    penalty_main(o, P, eps, bc, rhsr.data(), rhsi.data(), fr.data(), fi.data());
    if (cpenspecfilter) filter_column(o, fr.data(), fi.data());
    for (int k = 0; k < nz; ++k) {
      phi[o.idx(i, j, k)] = fr[k];
      phi[o.idx(i + 1, j, k)] = fi[k];
    }
  }
  // update (calcuvwt.f:826-901): ub = u* - dt i kx phi, vb likewise,
  // wb = w* - dt dphi/dz.  In calcuvwt_noslip.f the loop starts at k = 2 and
  // ub, vb, wb are calcuvwt's static local arrays: their k = 1 plane is never
  // written and stays zero.
  dpdz(o, phi.data(), dphidz.data());
  int kstart = noslip ? 1 : 0;
  for (int k = kstart; k < nz; ++k)
    for (int j = 0; j < o.ny; ++j)
      for (int ii = 0; ii < o.nxhp; ++ii) {
        size_t pr = o.idx(2 * ii, j, k), pi = pr + 1;
        bool lzero = (ii == 0 && j == 0);
        double dtx = o.dt * o.xw[ii], dty = o.dt * o.yw[j];
        o.ub[pr] = o.S[0][pr] - (0. * phi[pr] - dtx * phi[pi]);
        o.ub[pi] = o.S[0][pi] - (0. * phi[pi] + dtx * phi[pr]);
        o.vb[pr] = o.S[1][pr] - (0. * phi[pr] - dty * phi[pi]);
        o.vb[pi] = o.S[1][pi] - (0. * phi[pi] + dty * phi[pr]);
        if (lzero) {
          o.wb[pr] = 0.;
          o.wb[pi] = 0.;
        } else {
          o.wb[pr] = o.S[2][pr] - o.dt * dphidz[pr];
          o.wb[pi] = o.S[2][pi] - o.dt * dphidz[pi];
        }
      }
  // viscous solves (calcuvwt.f:247-591)
  const int ubot = noslip ? IDIR : INEU;
  const double xnudt = o.pp.xnu * o.dt, dtk = o.dt * o.pp.xkappa;
#pragma omp parallel for schedule(dynamic, 16)
  for (int c = 0; c < ncol; ++c) {
    int j = c / o.nxhp, ii = c % o.nxhp, i = 2 * ii;
    bool lzero = (ii == 0 && j == 0);
    Pen P(ns);
    double ak = o.xsq[ii] + o.ysq[j];
    std::vector<double> rhsr(nz), rhsi(nz), fr(nz), fi(nz);
    double eps = 1. / (ak + o.bdfv * o.facvel);
    BC bc{ubot, INEU, 0., 0., 0., 0.};
    // u
    penalty_setup(o, P, eps);
    for (int k = 0; k < nz; ++k) {
      rhsr[k] = -(o.ub[o.idx(i, j, k)] / xnudt);
      rhsi[k] = -(o.ub[o.idx(i + 1, j, k)] / xnudt);
    }
    penalty_main(o, P, eps, bc, rhsr.data(), rhsi.data(), fr.data(), fi.data());
    if (cpenspecfilter) filter_column(o, fr.data(), fi.data());
    if (lzero && o.pp.meanu_damping)
      for (int k = 0; k < nz; ++k) {
        double g = 1.0 - fzgaus(o.zg[k], o.pp.zcen, o.pp.xlen, o.pp.xbcrit);
        fr[k] = g * fr[k];
        fi[k] = g * fi[k];
      }
    for (int k = 0; k < nz; ++k) {
      o.F[0][o.idx(i, j, k)] = fr[k];
      o.F[0][o.idx(i + 1, j, k)] = fi[k];
    }
    // v
    penalty_setup(o, P, eps);
    for (int k = 0; k < nz; ++k) {
      rhsr[k] = -(o.vb[o.idx(i, j, k)] / xnudt);
      rhsi[k] = -(o.vb[o.idx(i + 1, j, k)] / xnudt);
    }
    penalty_main(o, P, eps, bc, rhsr.data(), rhsi.data(), fr.data(), fi.data());
    if (cpenspecfilter) filter_column(o, fr.data(), fi.data());
    for (int k = 0; k < nz; ++k) {
      o.F[1][o.idx(i, j, k)] = fr[k];
      o.F[1][o.idx(i + 1, j, k)] = fi[k];
    }
    // w (zero mode set to 0)
    if (lzero) {
      for (int k = 0; k < nz; ++k) fr[k] = fi[k] = 0.;
    } else {
      penalty_setup(o, P, eps);
      for (int k = 0; k < nz; ++k) {
        rhsr[k] = -(o.wb[o.idx(i, j, k)] / xnudt);
        rhsi[k] = -(o.wb[o.idx(i + 1, j, k)] / xnudt);
      }
      BC bw{IDIR, IDIR, 0., 0., 0., 0.};
      penalty_main(o, P, eps, bw, rhsr.data(), rhsi.data(), fr.data(), fi.data());
      if (cpenspecfilter) filter_column(o, fr.data(), fi.data());
    }
    for (int k = 0; k < nz; ++k) {
      o.F[2][o.idx(i, j, k)] = fr[k];
      o.F[2][o.idx(i + 1, j, k)] = fi[k];
    }
  }
  // density perturbation (calcuvwt.f:609-741)
#pragma omp parallel for schedule(dynamic, 16)
  for (int c = 0; c < ncol; ++c) {
    int j = c / o.nxhp, ii = c % o.nxhp, i = 2 * ii;
    Pen P(ns);
    double ak = o.xsq[ii] + o.ysq[j];
    std::vector<double> rhsr(nz), rhsi(nz), fr(nz), fi(nz);
    double eps = 1. / (ak + o.bdfv * o.fact);
    penalty_setup(o, P, eps);
    for (int k = 0; k < nz; ++k) {
      rhsr[k] = -(o.S[3][o.idx(i, j, k)] / dtk);
      rhsi[k] = -(o.S[3][o.idx(i + 1, j, k)] / dtk);
    }
    BC bt{INEU, INEU, 0., 0., 0., 0.};
    penalty_main(o, P, eps, bt, rhsr.data(), rhsi.data(), fr.data(), fi.data());
    if (cpenspecfilter) filter_column(o, fr.data(), fi.data());
    for (int k = 0; k < nz; ++k) {
      o.F[3][o.idx(i, j, k)] = fr[k];
      o.F[3][o.idx(i + 1, j, k)] = fi[k];
    }
  }
}

// penalty.f:714-775 interface_avg3d.
int interface_avg3d(Orc& o, double* f) {
  const double ct = 0.005, c1 = 0.5, c2 = 0.;
  horfft(o, f, 1, o.nz);
  int ic = 0;
  for (int i = 0; i < o.nxpp; ++i)
    for (int j = 0; j < o.ny; ++j)
      for (int ks = 1; ks < o.nsubd; ++ks) {
        int k = ks * o.nzloc, km = k - 1;
        double fsp = f[o.idx(i, j, k)], fsm = f[o.idx(i, j, km)];
        double favg2 = fsp + fsm;
        double c0 = std::fabs(fsp - fsm) / std::fabs(favg2);
        if (c0 > ct) {
          double ff = f[o.idx(i, j, km - 1)] * c1 + f[o.idx(i, j, km)] * c2 + f[o.idx(i, j, k)] * c2 +
                      f[o.idx(i, j, k + 1)] * c1;
          f[o.idx(i, j, km)] = ff;
          f[o.idx(i, j, k)] = ff;
          ++ic;
        }
      }
  horfft(o, f, -1, o.nz);
  return ic;
}

// various.f:665-987 maxcalc with the adaptive time step frozen: the state
// makes a horfft round trip; min/max/CFL and the uveltest probe are kept.
void maxcalc(Orc& o) {
  for (int q = 0; q < 4; ++q) horfft(o, o.F[q].data(), 1, o.nz);
  const double* u = o.F[0].data();
  const double* v = o.F[1].data();
  const double* w = o.F[2].data();
  const double* tp = o.F[3].data();
  // uveltest.dat probe u(32,1,10), u(32,1,50) (various.f:743-745)
  o.probe[0] = (o.nx >= 32 && o.nz >= 10) ? u[o.idx(31, 0, 9)] : 0.0;
  o.probe[1] = (o.nx >= 32 && o.nz >= 50) ? u[o.idx(31, 0, 49)] : 0.0;
  double umin = 0., umaxt = 0., vmin = 0., vmax = 0., wmin = 0., wmax = 0., tmin = 1., tmax = 0.;
  int kumin = 0, kumax = 0, kvmin = 0, kvmax = 0, kwmin = 0, kwmax = 0, ktmin = 0, ktmax = 0;
  double cflxmax = 0., cflymax = 0., cflzmax = 0.;
  int ic[9] = {0};
  double pi2 = 8.0 * std::atan(1.0);
  double dx = (pi2 / o.alpha) / o.nx, dy = (pi2 / o.beta) / o.ny;
  for (int i = 0; i < o.nx; ++i)
    for (int j = 0; j < o.ny; ++j)
      for (int ks = 0; ks < o.nsubd; ++ks)
        for (int kl = 0; kl < o.nzloc; ++kl) {
          int k = ks * o.nzloc + kl;
          int kg = ks * (o.nzloc - 1) + kl + 1;  // 1-based zf index
          size_t p = o.idx(i, j, k);
          if (u[p] >= umaxt) {
            umaxt = u[p] + o.pp.umax;
            kumax = k + 1;
          }
          if (u[p] <= umin) {
            umin = u[p];
            kumin = k + 1;
          }
          if (v[p] >= vmax) {
            vmax = v[p];
            kvmax = k + 1;
          }
          if (v[p] <= vmin) {
            vmin = v[p];
            kvmin = k + 1;
          }
          if (w[p] >= wmax) {
            wmax = w[p];
            kwmax = k + 1;
          }
          if (w[p] <= wmin) {
            wmin = w[p];
            kwmin = k + 1;
          }
          double rt = tp[p] + rhomean(o, o.zg[k]);
          if (rt >= tmax) {
            tmax = rt;
            ktmax = k + 1;
          }
          if (rt <= tmin) {
            tmin = rt;
            ktmin = k + 1;
          }
          double cflx = std::fabs((0.07 * 0.0 * 0.0 + u[p]) * o.dt / dx);
          double cfly = std::fabs(v[p] * o.dt / dy);
          double cflz;
          if (k + 1 == o.nz) {
            cflz = 0.;
          } else {
            // zf(0) is the word before zf(1) in COMMON: z(nz)
            double zkm1 = (kg - 1 >= 1) ? o.zf[kg - 1] : o.zg[o.nz - 1];
            double dz = o.zf[kg] - zkm1;
            cflz = std::fabs((w[p] * o.dt) / dz);
          }
          if (cflx >= cflxmax) {
            cflxmax = cflx;
            ic[0] = i + 1;
            ic[1] = j + 1;
            ic[2] = k + 1;
          }
          if (cfly >= cflymax) {
            cflymax = cfly;
            ic[3] = i + 1;
            ic[4] = j + 1;
            ic[5] = k + 1;
          }
          if (cflz >= cflzmax) {
            cflzmax = cflz;
            ic[6] = i + 1;
            ic[7] = j + 1;
            ic[8] = k + 1;
          }
        }
  double mm[8] = {umin, umaxt, vmin, vmax, wmin, wmax, tmin, tmax};
  int mi[8] = {kumin, kumax, kvmin, kvmax, kwmin, kwmax, ktmin, ktmax};
  std::memcpy(o.mm, mm, sizeof mm);
  std::memcpy(o.mm_idx, mi, sizeof mi);
  o.cfl[0] = cflxmax;
  o.cfl[1] = cflymax;
  o.cfl[2] = cflzmax;
  std::memcpy(o.cfl_idx, ic, sizeof ic);
  for (int q = 0; q < 4; ++q) horfft(o, o.F[q].data(), -1, o.nz);
}

extern "C" double orc_abvar1(double, double, double);
extern "C" double orc_abvar2(double, double, double);
extern "C" double orc_abvar3(double, double, double);
extern "C" double orc_bdfvarv(double, double, double);
extern "C" double orc_bdfvar1(double, double, double);
extern "C" double orc_bdfvar2(double, double, double);
extern "C" double orc_bdfvar3(double, double, double);

// various.f:892-937: the adaptive rule of maxcalc.  Tso (various.f:918,924) is
// a local of maxcalc without SAVE that is read before any store to it, and
// the store does not outlive the call; the reference's recorded run
// (dtchange.dat: 2.1 0.125, 2.725 0.15625, ... from dtin = 0.1) changes dt
// exactly when the count from Tso = 0 exceeds 20, which is what is kept here.
bool dt_rule(double cflxmax, double cflzmax, double t, double& dt, double xomega, double& cdt) {
  const double cflxmax_lim = 0.16, cflzmax_lim = 0.7, cflzmin_lim = 0.1;
  const bool change_dt = (cflzmax > cflzmax_lim) || (cflzmax < cflzmin_lim) || (cflxmax > cflxmax_lim);
  const double pi2 = 8.0 * std::atan(1.0);
  const double Tlim = pi2 / (xomega * 50.);
  const double Tso = 0.0;
  const double q = (t - Tso) / dt;  // Nst = INT(q): truncation toward zero
  const long long Nst = q >= 9.0e18 ? 9000000000000000000LL : q <= -9.0e18 ? -1LL : (long long)q;
  if (Nst > 20 && change_dt) {
    if (cflzmax < cflzmin_lim) cdt = std::max(0.8, dt / Tlim);
    if ((cflzmax > cflzmax_lim) || (cflxmax > cflxmax_lim)) cdt = 1.25;
    dt = dt / cdt;
    return true;
  }
  return false;
}

// various.f:938-970: new dt, the coefficients of the step that follows (one
// step of the new dt and two of the old in the history), facvel and fact
void adapt_dt(Orc& o) {
  const Wave wv = wave_params(o);
  if (!dt_rule(o.cfl[0], o.cfl[2], o.t, o.dt, wv.xomega, o.cdt)) return;
  const double dt1 = o.dt, dt2 = o.cdt * o.dt, dt3 = o.cdt * o.dt;
  o.fac1 = orc_abvar1(dt1, dt2, dt3);
  o.fac2 = orc_abvar2(dt1, dt2, dt3);
  o.fac3 = orc_abvar3(dt1, dt2, dt3);
  o.bdf1 = orc_bdfvar1(dt1, dt2, dt3);
  o.bdf2 = orc_bdfvar2(dt1, dt2, dt3);
  o.bdf3 = orc_bdfvar3(dt1, dt2, dt3);
  o.bdfv = orc_bdfvarv(dt1, dt2, dt3);
  o.fact = 1. / (o.pp.xkappa * o.dt);
  o.facvel = 1. / (o.pp.xnu * o.dt);
  o.ivardt = 1;
  o.idtstep = 0;
}

// solver.f:136-222: the animation dump of convec.  Physical fields by
// horfft +1 on copies.  The reference reads u(i,j,k) with j = ny+1, the value
// the y loop of solver.f:82-100 leaves: u(i,1,k+1), and for k = nz the first
// row of the array after it in COMMON /flow/ (u -> v, w -> temp, temp -> un).
// the animdump.log line (solver.f:212-215): list-directed t (15 significant
// digits, F form), I12 counters, a blank before a character item after a number
std::string animdump_line(double t, int n, int istep) {
  char e[40], num[64], tail[128];
  std::snprintf(e, sizeof e, "%.14e", t);
  const int ex = std::atoi(std::strchr(e, 'e') + 1);
  std::snprintf(num, sizeof num, "%.*f", ex >= 14 ? 0 : 14 - ex, t);
  std::snprintf(tail, sizeof tail, "      vortanimout_%12d .datat step=%12d\n", n, istep);
  return std::string(" Animation data dumped out at time   ") + num + tail;
}

void anim_dump(Orc& o) {
  const size_t row = o.nxpp, plane = (size_t)o.nxpp * o.ny;
  std::vector<double> ph[4];
  for (int q = 0; q < 4; ++q) {
    ph[q] = o.F[q];
    if (q == 2)  // wc(1,1,k) = 0 at the top of convec (solver.f:64-67)
      for (int k = 0; k < o.nz; ++k) ph[q][o.idx(0, 0, k)] = ph[q][o.idx(1, 0, k)] = 0.0;
    horfft(o, ph[q].data(), 1, o.nz);
  }
  // COMMON /flow/ from u on: u v w temp (physical here) then un (spectral)
  auto flow = [&](int arr, size_t idx) -> double {
    const size_t n = o.ntot;
    while (idx >= n) { idx -= n; ++arr; }
    return arr < 4 ? ph[arr][idx] : o.Fn[arr - 4][idx];
  };
  char name[32];
  std::snprintf(name, sizeof name, "vortanimout_%05d.dat", o.ianimc);
  const std::string path = o.anim_dir.empty() ? std::string(name) : o.anim_dir + "/" + name;
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) return;
  std::fprintf(f, " ZONE F=POINT, I=%12d , J=%12d\n", o.nx, o.nz);
  const double rg = rhograd(o);
  for (int ks = 0; ks < o.nsubd; ++ks)
    for (int kl = 0; kl < o.nzloc; ++kl) {
      const int k = ks * o.nzloc + kl;
      const double zz = o.zg[k];
      for (int i = 0; i < o.nx; ++i) {
        const size_t idx = (size_t)i + row * (size_t)o.ny + plane * (size_t)k;  // (i, ny+1, k)
        const double u = flow(0, idx), w = flow(2, idx), tt = flow(3, idx);
        std::fprintf(f, " ");
        for (double v : {o.xg[i], zz, u, w, tt, tt + (1. + rg * zz)}) std::fprintf(f, "%25.16f   ", v);
        std::fprintf(f, "\n");
      }
    }
  std::fclose(f);
  FILE* lf = std::fopen((o.anim_dir.empty() ? std::string("animdump.log") : o.anim_dir + "/animdump.log").c_str(), "a");
  if (lf) {
    std::fputs(animdump_line(o.t, o.ianimc, o.istep).c_str(), lf);
    std::fclose(lf);
  }
}

// Fortran E12.6 for the non-negative values of the spectra: 0.dddddd E+ee
static std::string e12_6_nonneg(double v) {
  if (v == 0.0) return "0.000000E+00";
  char m[40], out[40];
  std::snprintf(m, sizeof m, "%.5e", v);  // d.ddddde+XX: 6 significant digits
  const int e = std::atoi(m + 8) + 1;
  if (std::abs(e) <= 99) std::snprintf(out, sizeof out, "0.%c%.5sE%c%02d", m[0], m + 2, e < 0 ? '-' : '+', std::abs(e));
  else std::snprintf(out, sizeof out, "0.%c%.5s%c%03d", m[0], m + 2, e < 0 ? '-' : '+', std::abs(e));
  return out;
}

// filtering.f:1110-1221 (speclegencalc) on a copy of one field: physical
// space, the x row at y index nyh (1-based), per subdomain the mean over x of
// |a_k|, then the file speclegen<c><t>.dat, FORMAT (1x,I2,2x,10(e12.6,2x)).
void speclegen(Orc& o, char c, const std::vector<double>& field) {
  std::vector<double> fin = field;
  horfft(o, fin.data(), 1, o.nz);
  const int N = o.nzloc, nzm = N - 1, j = o.nyh - 1;
  std::vector<double> specout((size_t)o.nsubd * N, 0.0), faux(N), a(N);
  for (int ks = 0; ks < o.nsubd; ++ks) {
    for (int i = 0; i < o.nx; ++i) {
      for (int kloc = 0; kloc < N; ++kloc) faux[kloc] = fin[o.idx(i, j, ks * N + kloc)];
      for (int k = 0; k <= nzm; ++k) {
        double sum = 0.;
        for (int k1 = 0; k1 < N; ++k1) sum = sum + o.wg[k1] * faux[k1] * o.alpol[(size_t)k * N + k1];
        a[k] = (k == nzm) ? 0.5 * nzm * sum : (k + 0.5) * sum;
      }
      for (int kloc = 0; kloc < N; ++kloc) specout[(size_t)ks * N + kloc] = specout[(size_t)ks * N + kloc] + std::fabs(a[kloc]);
    }
    for (int kloc = 0; kloc < N; ++kloc) specout[(size_t)ks * N + kloc] = specout[(size_t)ks * N + kloc] / o.nx;
  }
  // file name: 'speclegen' // c // t in F5.3 (F6.3 .. F8.3 by nint(t)) // '.dat'
  const long nt = std::lround(o.t);
  const int w = nt >= 1000 ? 8 : nt >= 100 ? 7 : nt >= 10 ? 6 : 5;
  char tb[64];
  std::snprintf(tb, sizeof tb, "%.3f", o.t);
  std::string ts(tb);
  ts = (int)ts.size() > w ? std::string(w, '*') : std::string(w - ts.size(), ' ') + ts;
  const std::string name = std::string("speclegen") + c + ts + ".dat";
  const std::string path = o.leg_dir.empty() ? name : o.leg_dir + "/" + name;
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) return;
  for (int kloc = 0; kloc < N; ++kloc) {
    std::fprintf(f, " %2d  ", kloc + 1);
    for (int ks = 0; ks < o.nsubd; ++ks) {
      if (ks > 0) std::fputs(ks % 10 == 0 ? "\n" : "  ", f);  // format reversion after 10 values
      std::fprintf(f, "%12s", e12_6_nonneg(specout[(size_t)ks * N + kloc]).c_str());
    }
    std::fputs("\n", f);
  }
  std::fclose(f);
}

// main.f:653-1066, one step with istart=0; maxcalc's adaptive step when
// imaxcalc = 1 (the reference hard-codes 1, main.f:47), dt fixed otherwise.
void step(Orc& o) {
  o.istep += 1;
  int istep = o.istep;
  maxcalc(o);
  if (o.pp.imaxcalc == 1) adapt_dt(o);
  if (o.ivardt == 1) o.idtstep = o.idtstep + 1;  // main.f:660-662
  if (o.dtanim > 0 && (o.t - o.tdump) >= o.dtanim) {  // solver.f:141-142
    o.tdump = o.t;
    o.ianimc = o.ianimc + 1;
    anim_dump(o);
  }
  convec(o);
  bool ldtadapt = (o.ivardt == 1) && (o.idtstep < 2);  // main.f:741
  if (istep < 2 && o.istart == 0) {
    o.fac1 = 2.;
    o.fac2 = -1.;
    o.fac3 = 0.;
    o.bdf1 = 2.;
    o.bdf2 = -0.5;
    o.bdf3 = 0.;
  } else if (istep >= 2 && !ldtadapt) {
    o.fac1 = 3.;
    o.fac2 = -3.;
    o.fac3 = 1.;
    o.bdf1 = 3.;
    o.bdf2 = -1.5;
    o.bdf3 = 1. / 3.;
  } else {  // main.f:716-730 (restart, istep = 1) and 760-775
    const double dt1 = o.dt, dt2 = o.dt, dt3 = o.cdt * o.dt;
    o.fac1 = orc_abvar1(dt1, dt2, dt3);
    o.fac2 = orc_abvar2(dt1, dt2, dt3);
    o.fac3 = orc_abvar3(dt1, dt2, dt3);
    o.bdf1 = orc_bdfvar1(dt1, dt2, dt3);
    o.bdf2 = orc_bdfvar2(dt1, dt2, dt3);
    o.bdf3 = orc_bdfvar3(dt1, dt2, dt3);
  }
  for (int q = 0; q < 4; ++q) o.S[q] = o.F[q];
  bool cpen = (o.pp.ispecfilterexp == 1) && (istep % o.pp.nspecfilterexp == 0);
  calcuvwt(o, cpen);
  ldtadapt = (o.ivardt == 1) && (o.idtstep < 2);  // main.f:832
  if (istep < 2) {
    if (o.istart == 0) {
      o.bdfv = 1.5;
    } else {  // main.f:820-826
      const double dt1 = o.dt, dt2 = o.dt, dt3 = o.cdt * o.dt;
      o.bdfv = orc_bdfvarv(dt1, dt2, dt3);
    }
  } else if (!ldtadapt) {
    o.bdfv = 11. / 6.;
  } else {  // main.f:846-852
    const double dt1 = o.dt, dt2 = o.dt, dt3 = o.cdt * o.dt;
    o.bdfv = orc_bdfvarv(dt1, dt2, dt3);
    o.cdt = 1.;
    o.ivardt = 0;
  }
  o.t = o.t + o.dt;
  if (o.nlegspec > 0 && istep % o.nlegspec == 0) {  // main.f:905-910
    speclegen(o, 'u', o.F[0]);
    speclegen(o, 'v', o.F[1]);
    speclegen(o, 'w', o.F[2]);
    speclegen(o, 'T', o.F[3]);
  }
  if (o.pp.navgintrfc > 0 && istep % o.pp.navgintrfc == 0)
    for (int q = 0; q < 4; ++q) o.avg_count[q] = interface_avg3d(o, o.F[q].data());
}

// Mode-1 wave + seeded noise (new init; see iw_init_mode1 in the header).
void init_mode1(Orc& o, double A, double anoise, uint64_t seed) {
  Wave wv = wave_params(o);
  for (int q = 0; q < 4; ++q) {
    std::fill(o.F[q].begin(), o.F[q].end(), 0.0);
    std::fill(o.Fn[q].begin(), o.Fn[q].end(), 0.0);
    std::fill(o.Fnm[q].begin(), o.Fnm[q].end(), 0.0);
    std::fill(o.S[q].begin(), o.S[q].end(), 0.0);
    std::fill(o.Sn[q].begin(), o.Sn[q].end(), 0.0);
    std::fill(o.Snm[q].begin(), o.Snm[q].end(), 0.0);
  }
  double kx = wv.xkcrit, m = wv.xmcrit, om = wv.xomega;
  double rc = (o.pp.rho0 * bruntz(o) * bruntz(o)) / o.pp.grav;
  for (int k = 0; k < o.nz; ++k)
    for (int j = 0; j < o.ny; ++j)
      for (int i = 0; i < o.nx; ++i) {
        double x = o.xg[i], z = o.zg[k];
        size_t p = o.idx(i, j, k);
        o.F[0][p] = -(A / kx) * m * std::cos(m * z) * std::sin(kx * x);
        o.F[2][p] = A * std::sin(m * z) * std::cos(kx * x);
        o.F[3][p] = -(A / om) * rc * std::sin(m * z) * std::sin(kx * x);
      }
  // xorshift64 (shift triple 21, 35, 4 as in random/random.f:62-80), seeded
  uint64_t s = seed ? seed : 0x9E3779B97F4A7C15ULL;
  for (int k = 0; k < o.nz; ++k) {
    if (!(o.zg[k] < 0.2 * o.pp.zlen)) continue;
    for (int j = 0; j < o.ny; ++j)
      for (int i = 0; i < o.nx; ++i)
        for (int q = 0; q < 3; ++q) {
          s ^= s << 21;
          s ^= s >> 35;
          s ^= s << 4;
          double r = (double)(int64_t)s * 5.42101086242752217e-20 + 0.5;  // (0,1)
          o.F[q][o.idx(i, j, k)] += anoise * (2.0 * r - 1.0);
        }
  }
  for (int q = 0; q < 4; ++q) horfft(o, o.F[q].data(), -1, o.nz);
  o.t = 0.0;
  o.istep = 0;
  o.cdt = 1.;
  o.ivardt = 0;
  o.idtstep = 0;
  o.istart = 0;
  o.fac1 = 1.;
  o.fac2 = o.fac3 = 0.;
  o.bdf1 = 1.;
  o.bdf2 = o.bdf3 = 0.;
  o.bdfv = 1.;
}

// KE and dissipation (postp.f:415-732 definitions: plain grid sums over
// i=1..nx, all j, k=2..nz, without mean removal).
void diag_energy(Orc& o, double* out) {
  std::vector<double> f[4], g[12];
  for (int q = 0; q < 4; ++q) f[q] = o.F[q];
  for (auto& x : g) x.assign(o.ntot, 0.0);
  for (int q = 0; q < 3; ++q) {
    dpdz(o, f[q].data(), g[3 * q + 2].data());
    for (int k = 0; k < o.nz; ++k)
      for (int j = 0; j < o.ny; ++j)
        for (int ii = 0; ii < o.nxhp; ++ii) {
          size_t pr = o.idx(2 * ii, j, k), pi = pr + 1;
          g[3 * q][pr] = -(o.xw[ii] * f[q][pi]);
          g[3 * q][pi] = o.xw[ii] * f[q][pr];
          g[3 * q + 1][pr] = -(o.yw[j] * f[q][pi]);
          g[3 * q + 1][pi] = o.yw[j] * f[q][pr];
        }
  }
  for (int q = 0; q < 3; ++q) horfft(o, f[q].data(), 1, o.nz);
  for (int q = 0; q < 9; ++q) horfft(o, g[q].data(), 1, o.nz);
  double ke = 0, eps = 0, wsum = 0;
  long wcnt = 0;
  for (int k = 1; k < o.nz; ++k)
    for (int j = 0; j < o.ny; ++j)
      for (int i = 0; i < o.nx; ++i) {
        size_t p = o.idx(i, j, k);
        ke += f[0][p] * f[0][p] + f[1][p] * f[1][p] + f[2][p] * f[2][p];
        double e = 0;
        for (int q = 0; q < 9; ++q) e += g[q][p] * g[q][p];
        eps += e;
      }
  for (int k = 0; k < o.nz; ++k) {
    if (!(o.zg[k] < 0.2 * o.pp.zlen)) continue;
    for (int j = 0; j < o.ny; ++j)
      for (int i = 0; i < o.nx; ++i) {
        double wv = f[2][o.idx(i, j, k)];
        wsum += wv * wv;
        ++wcnt;
      }
  }
  out[0] = 0.5 * ke;
  out[1] = o.pp.xnu * eps;
  out[2] = wcnt ? std::sqrt(wsum / wcnt) : 0.0;
}

// postp.f:9-70 (postp) on copies of the state, with umeancalc
// (postp.f:129-213), dpdzyzplane (postp.f:984-1020), dudymeancalc
// (postp.f:237-298), perturbcalc (postp.f:300-330) and energycalc_postp
// (postp.f:415-732).  e18: one energy.dat line; w18: one energy_wake.dat line
// (the wake radii are never set, wakelengthcalc being commented out at
// postp.f:36-38, so no point is inside the wake and only tkemean is nonzero).
void postp(Orc& o, double* e18, double* w18) {
  const int nx = o.nx, ny = o.ny, nz = o.nz, N = o.nzloc;
  std::vector<double> u = o.F[0], v = o.F[1], w = o.F[2], tp = o.F[3];
  for (auto* f : {&u, &v, &w, &tp}) horfft(o, f->data(), 1, nz);
  // umeancalc: x means for k = 2..nz
  std::vector<double> umean((size_t)ny * nz, 0.0), dumeandz((size_t)ny * nz, 0.0), dumeandy((size_t)ny * nz, 0.0);
  for (int k = 1; k < nz; ++k)
    for (int j = 0; j < ny; ++j) {
      double s = 0.;
      for (int i = 0; i < nx; ++i) s = s + u[o.idx(i, j, k)];
      umean[(size_t)j * nz + k] = s / nx;
    }
  // dudzmeancalc: dpdzcol per y and subdomain
  for (int j = 0; j < ny; ++j)
    for (int ks = 0; ks < o.nsubd; ++ks) {
      double a[IW_MAX_NZLOC], b[IW_MAX_NZLOC];
      for (int kl = 0; kl < N; ++kl) a[kl] = umean[(size_t)j * nz + ks * N + kl];
      dpdzcol(o, a, b, o.pp.zh[ks]);
      for (int kl = 0; kl < N; ++kl) dumeandz[(size_t)j * nz + ks * N + kl] = b[kl];
    }
  // dudymeancalc: real Fourier series in y times i ky; the imaginary Nyquist
  // coefficient is dropped by the real inverse transform
  if (ny > 1) {
    const double pi2 = 8.0 * std::atan(1.0);
    std::vector<cd> zin(ny), zout(ny), spec(ny);
    for (int k = 0; k < nz; ++k) {
      for (int j = 0; j < ny; ++j) zin[j] = cd(umean[(size_t)j * nz + k], 0.0);
      o.fy.run(zin.data(), zout.data(), false);
      std::fill(spec.begin(), spec.end(), cd(0.0, 0.0));
      for (int m = 1; m < ny / 2; ++m) {
        const cd a = zout[m] / (double)ny * cd(0.0, m * (pi2 / o.pp.ylen));
        spec[m] = a;
        spec[ny - m] = std::conj(a);
      }
      o.fy.run(spec.data(), zout.data(), true);
      for (int j = 0; j < ny; ++j) dumeandy[(size_t)j * nz + k] = zout[j].real();
    }
  }
  // perturbcalc
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) u[o.idx(i, j, k)] = u[o.idx(i, j, k)] - umean[(size_t)j * nz + k];
  // energycalc_postp: gradients in spectral space, back to physical space
  for (auto* f : {&u, &v, &w, &tp}) horfft(o, f->data(), -1, nz);
  std::vector<double>* fl[4] = {&u, &v, &w, &tp};
  std::vector<double> g[12];
  for (auto& x : g) x.assign(o.ntot, 0.0);
  for (int q = 0; q < 4; ++q) {
    const std::vector<double>& f = *fl[q];
    dpdz(o, f.data(), g[3 * q + 2].data());
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int ii = 0; ii < o.nxhp; ++ii) {
          const size_t pr = o.idx(2 * ii, j, k), pi = pr + 1;
          g[3 * q][pr] = -(o.xw[ii] * f[pi]);
          g[3 * q][pi] = o.xw[ii] * f[pr];
          g[3 * q + 1][pr] = -(o.yw[j] * f[pi]);
          g[3 * q + 1][pi] = o.yw[j] * f[pr];
        }
  }
  for (auto* f : {&u, &v, &w, &tp}) horfft(o, f->data(), 1, nz);
  for (auto& x : g) horfft(o, x.data(), 1, nz);
  double tketot = 0, u1 = 0, u2 = 0, u3 = 0, prody = 0, prodz = 0, bflux = 0, tempvar = 0, eps = 0, chi = 0, tkemean = 0;
  for (int k = 1; k < nz; ++k)
    for (int j = 0; j < ny; ++j) {
      for (int i = 0; i < nx; ++i) {
        const size_t p = o.idx(i, j, k);
        const double uu = u[p], vv = v[p], ww = w[p], tt = tp[p];
        tketot = tketot + (uu * uu + vv * vv + ww * ww);
        u1 = u1 + uu * uu;
        u2 = u2 + vv * vv;
        u3 = u3 + ww * ww;
        prody = prody - dumeandy[(size_t)j * nz + k] * (uu * vv);
        prodz = prodz - dumeandz[(size_t)j * nz + k] * (uu * ww);
        bflux = bflux + ww * tt;
        tempvar = tempvar + tt * tt;
        for (int q = 0; q < 9; ++q) eps = eps + g[q][p] * g[q][p];
        for (int q = 9; q < 12; ++q) chi = chi + g[q][p] * g[q][p];
      }
      tkemean = tkemean + umean[(size_t)j * nz + k] * umean[(size_t)j * nz + k];
    }
  const double ra = 0.0, pr = o.pp.xnu;  // ra: start-up value (main.f:577-580); pr = xnu (main.f:428)
  tketot = tketot * 0.5;
  tkemean = tkemean * 0.5 * nx;
  bflux = bflux * ra * pr;
  eps = eps * pr;
  chi = chi * o.pp.xkappa;
  const double tt = o.t - o.tstart;
  const double e[18] = {tt,  tt * o.pp.brunt, tketot, u1, u2, u3, prody, prodz, prody + prodz, bflux, eps, 0.0,
                        eps + 0.0, chi, 0.0, 0.0 + chi, tkemean, tempvar};
  std::memcpy(e18, e, sizeof e);
  for (int n = 0; n < 18; ++n) w18[n] = 0.0;
  w18[0] = e[0];
  w18[1] = e[1];
  w18[16] = tkemean;
}

std::string g_err;

}  // namespace

// ---------------------------------------------------------------------------
// C API for the Python test harness (ctypes).
// ---------------------------------------------------------------------------
extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

void* orc_create(const iw_dims* d, const iw_params* p) {
  if (!d || !p || d->nx < 2 || d->nx % 2 || d->ny < 1 || (d->ny > 1 && d->ny % 2) || d->nzloc < 3 ||
      d->nzloc > IW_MAX_NZLOC || d->nsubd < 1 || d->nsubd > IW_MAX_SUBD) {
    g_err = "invalid dims";
    return nullptr;
  }
  Orc* o = new Orc();
  o->dm = *d;
  o->pp = *p;
  o->nx = d->nx;
  o->ny = d->ny;
  o->nzloc = d->nzloc;
  o->nsubd = d->nsubd;
  o->nz = d->nzloc * d->nsubd;
  o->nzm = d->nzloc - 1;
  o->nxpp = d->nx + 2;
  o->nxh = d->nx / 2;
  o->nxhp = o->nxh + 1;
  o->nyh = d->ny / 2;
  o->ndims = d->ny > 1 ? 3 : 2;
  o->ntot = (size_t)o->nxpp * o->ny * o->nz;
  double pi2 = 8.0 * std::atan(1.0);
  o->alpha = pi2 / p->xlen;
  o->beta = pi2 / p->ylen;
  o->scaley = 1. / (double)o->ny;
  o->dt = p->dt;
  o->fact = 1. / (p->xkappa * o->dt);
  o->facvel = 1. / (p->xnu * o->dt);
  for (int q = 0; q < 4; ++q) {
    o->F[q].assign(o->ntot, 0.0);
    o->Fn[q] = o->Fnm[q] = o->S[q] = o->Sn[q] = o->Snm[q] = o->F[q];
  }
  o->ub.assign(o->ntot, 0.0);
  o->vb = o->wb = o->ub;
  o->wnl.assign((size_t)o->nxpp * o->ny * 2, 0.0);
  o->wviscrot = o->wnl;
  o->pen0 = new Pen(o->nsubd);
  o->pen0->omega = 2. / (double)((o->nzloc + 1) * (o->nzloc + 2));
  setup(*o);
  return o;
}

void orc_destroy(void* h) {
  Orc* o = (Orc*)h;
  delete o->pen0;
  delete o;
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : 1);
#else
  (void)n;
#endif
}

int orc_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_fourier_scale(void* h, int on) { ((Orc*)h)->fourier_scale = on != 0; }

void orc_set_cache(void* h, int on) {
  Orc* o = (Orc*)h;
  o->cache_on = on != 0;
  o->cache.clear();
}

// tables: zpts(nzloc), wg(nzloc), d(nzloc^2 row major), d2, alpol, z(nz), sigma(nzloc)
void orc_tables(void* h, double* zpts, double* wg, double* d, double* d2, double* alpol, double* z, double* sigma) {
  Orc* o = (Orc*)h;
  size_t N = o->nzloc;
  if (zpts) std::memcpy(zpts, o->zpts.data(), N * 8);
  if (wg) std::memcpy(wg, o->wg.data(), N * 8);
  if (d) std::memcpy(d, o->dmat.data(), N * N * 8);
  if (d2) std::memcpy(d2, o->d2mat.data(), N * N * 8);
  if (alpol) std::memcpy(alpol, o->alpol.data(), N * N * 8);
  if (z) std::memcpy(z, o->zg.data(), (size_t)o->nz * 8);
  if (sigma) std::memcpy(sigma, o->leg_sigma.data(), N * 8);
}

// level 0: u,v,w,temp at n; 1: n-1; 2: n-2; 3: NL at n-1; 4: NL at n-2
void orc_set_state(void* h, int level, const double* uvwt) {
  Orc* o = (Orc*)h;
  std::vector<double>* L = level == 0 ? o->F : level == 1 ? o->Fn : level == 2 ? o->Fnm : level == 3 ? o->Sn : o->Snm;
  for (int q = 0; q < 4; ++q) std::memcpy(L[q].data(), uvwt + q * o->ntot, o->ntot * 8);
}
void orc_get_state(void* h, int level, double* uvwt) {
  Orc* o = (Orc*)h;
  std::vector<double>* L = level == 0 ? o->F : level == 1 ? o->Fn : level == 2 ? o->Fnm : level == 3 ? o->Sn : o->Snm;
  for (int q = 0; q < 4; ++q) std::memcpy(uvwt + q * o->ntot, L[q].data(), o->ntot * 8);
}
// scalars: t, istep, fac1..3, bdf1..3, bdfv
void orc_get_scalars(void* h, double* out) {
  Orc* o = (Orc*)h;
  double v[9] = {o->t, (double)o->istep, o->fac1, o->fac2, o->fac3, o->bdf1, o->bdf2, o->bdf3, o->bdfv};
  std::memcpy(out, v, sizeof v);
}
void orc_set_scalars(void* h, const double* in) {
  Orc* o = (Orc*)h;
  o->t = in[0];
  o->istep = (int)in[1];
  o->fac1 = in[2];
  o->fac2 = in[3];
  o->fac3 = in[4];
  o->bdf1 = in[5];
  o->bdf2 = in[6];
  o->bdf3 = in[7];
  o->bdfv = in[8];
  o->cdt = 1.;
  o->ivardt = 0;
  o->idtstep = 0;
  o->istart = 0;
}

void orc_init_mode1(void* h, double A, double anoise, uint64_t seed) { init_mode1(*(Orc*)h, A, anoise, seed); }

// current dt and the adaptive state: dt, cdt, ivardt, idtstep
void orc_get_dt(void* h, double* out4) {
  Orc* o = (Orc*)h;
  double v[4] = {o->dt, o->cdt, (double)o->ivardt, (double)o->idtstep};
  std::memcpy(out4, v, sizeof v);
}
// the rule alone (dt_rule): returns 1 and the new dt and cdt on a change
int orc_dt_rule(double cflx, double cflz, double t, double dt, double xomega, double* dt_new, double* cdt) {
  double d = dt, c = 1.;
  if (!dt_rule(cflx, cflz, t, d, xomega, c)) return 0;
  *dt_new = d;
  *cdt = c;
  return 1;
}

// ---------------------------------------------------------------------------
// Restart files.  output.f:2-117 writes them, restart.f:2-126 reads them and
// main.f:555-632 sets up the steps after a read.  ifort unformatted
// sequential: every record framed by its byte count (4-byte little-endian
// integer) before and after; REAL*8 (-autodouble) and INTEGER*4 items.
// Setup tables the oracle does not keep (dalpol, d3, atpz/btpz/ctpz), the
// boundary arrays the step never reads (tubc/tbbc, uw/vw/ww), solks and the
// soliton fields (never set: wavesetup is not called) are written as 0; past
// nxhp, record 5 holds 0 (the reference writes past xw's bound there).  A
// 50th record, which restart.f never reads, carries the step counter, the
// adaptive and restart state and the coefficients (exact continuation).
// ---------------------------------------------------------------------------
struct RstRecs {
  std::vector<std::vector<char>> r;
  void open() { r.emplace_back(); }
  void d(double v) { r.back().insert(r.back().end(), (const char*)&v, (const char*)&v + 8); }
  void i(int32_t v) { r.back().insert(r.back().end(), (const char*)&v, (const char*)&v + 4); }
  void zeros(size_t n8) { r.back().insert(r.back().end(), 8 * n8, (char)0); }
  void field(const std::vector<double>& f) { r.back().insert(r.back().end(), (const char*)f.data(), (const char*)(f.data() + f.size())); }
};
static std::vector<size_t> rst_sizes(const Orc& o) {  // bytes of records 1..49, output.f:26-108
  const size_t nx = o.nx, ny = o.ny, nz = o.nz, N = o.nzloc, ns = o.nsubd, nxpp = o.nxpp;
  const size_t nz2 = ns * (N - 1) + 1;
  std::vector<size_t> b = {8, 16, 36, 16, 16 * nx, 16 * ny, 8 * nx, 8 * ny, 8 * nz, 8 * nz2, 20 * ns, 8,
                           8 * N * N, 8 * N * N, 8 * N, 8 * N, 8 * N * N, 8 * N * N, 8 * N * N, 24 * nz,
                           16 * nxpp * ny, 96 * nxpp * ny, 8, 8, 16 * nxpp * nz, 16 * nxpp * nz, 16 * nxpp * nz,
                           8 * nxpp * nz, 16 * nxpp * nz};
  for (int q = 0; q < 20; ++q) b.push_back(8 * o.ntot);
  return b;
}

int orc_write_restart(void* h, const char* path) {
  Orc& o = *(Orc*)h;
  const int N = o.nzloc, ns = o.nsubd;
  RstRecs w;
  w.open(); w.d(o.t);                                    // output.f:26
  w.open(); w.d(o.pp.xnu); w.d(0.0);                     // :27, pr = xnu (main.f:428), ra = 0
  w.open();                                              // :28
  for (int32_t v : {o.nx, o.ny, o.nz, N - 1, o.nxpp * o.ny, (int32_t)o.ntot, ns, N, 1}) w.i(v);
  w.open(); w.d(o.alpha); w.d(o.beta);                   // :29
  w.open();                                              // :30
  for (int i = 0; i < o.nx; ++i) {
    w.d(i < o.nxhp ? o.xw[i] : 0.0);
    w.d(i < o.nxhp ? o.xsq[i] : 0.0);
  }
  w.open();                                              // :31
  for (int j = 0; j < o.ny; ++j) { w.d(o.yw[j]); w.d(o.ysq[j]); }
  w.open(); for (double v : o.xg) w.d(v);                // :32
  w.open(); for (double v : o.yg) w.d(v);                // :33
  w.open(); for (double v : o.zg) w.d(v);                // :34
  w.open(); for (int k = 1; k <= ns * (N - 1) + 1; ++k) w.d(o.zf[k]);  // :35
  w.open(); for (int k = 0; k < ns; ++k) { w.d(o.pp.z0[k]); w.d(o.pp.zh[k]); w.i(1); }  // :36
  w.open(); w.d(o.pp.zlen * (1. / ns));                  // :37, setup.f:281,289
  w.open(); for (int k = 0; k < N; ++k) for (int j = 0; j < N; ++j) w.d(o.alpol[(size_t)j * N + k]);  // :38
  w.open(); w.zeros((size_t)N * N);                      // :39 dalpol
  w.open(); for (double v : o.zpts) w.d(v);              // :40
  w.open(); for (double v : o.wg) w.d(v);                // :41
  w.open(); for (int j = 0; j < N; ++j) for (int i = 0; i < N; ++i) w.d(o.dmat[(size_t)i * N + j]);   // :42
  w.open(); for (int j = 0; j < N; ++j) for (int i = 0; i < N; ++i) w.d(o.d2mat[(size_t)i * N + j]);  // :43
  w.open(); w.zeros((size_t)N * N);                      // :44 d3
  w.open(); w.zeros(3 * (size_t)o.nz);                   // :45
  w.open(); w.zeros(2 * (size_t)o.nxpp * o.ny);          // :46
  w.open(); w.zeros(12 * (size_t)o.nxpp * o.ny);         // :47-49
  w.open(); w.d(o.pp.umax);                              // :52
  w.open(); w.d(0.0);                                    // :53 solks
  for (size_t n : {2, 2, 2, 1, 2}) { w.open(); w.zeros(n * (size_t)o.nxpp * o.nz); }  // :54-58
  for (auto* L : {o.F, o.Fn, o.Fnm, o.Sn, o.Snm})       // :66-105
    for (int q = 0; q < 4; ++q) { w.open(); w.field(L[q]); }
  w.open();
  for (int32_t v : {0x32425749, 1, o.istep, o.ivardt, o.idtstep, o.istart}) w.i(v);
  for (double v : {o.dt, o.cdt, o.fac1, o.fac2, o.fac3, o.bdf1, o.bdf2, o.bdf3, o.bdfv}) w.d(v);
  FILE* f = std::fopen(path, "wb");
  if (!f) { g_err = std::string("cannot open ") + path; return 1; }
  bool ok = true;
  for (const auto& r : w.r) {
    const uint32_t m = (uint32_t)r.size();
    ok = ok && std::fwrite(&m, 4, 1, f) == 1 && (r.empty() || std::fwrite(r.data(), 1, r.size(), f) == r.size()) &&
         std::fwrite(&m, 4, 1, f) == 1;
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) { g_err = std::string("write error on ") + path; return 1; }
  return 0;
}

// mode 0: exact continuation (needs the 50th record); 1: main.f istart = 1
int orc_read_restart(void* h, const char* path, int mode, double cdtin) {
  Orc& o = *(Orc*)h;
  FILE* f = std::fopen(path, "rb");
  if (!f) { g_err = std::string("cannot open ") + path; return 1; }
  std::vector<std::vector<char>> recs;
  for (;;) {
    uint32_t m = 0, m2 = 0;
    if (std::fread(&m, 4, 1, f) != 1) break;
    std::vector<char> r(m);
    if ((m && std::fread(r.data(), 1, m, f) != m) || std::fread(&m2, 4, 1, f) != 1 || m2 != m) {
      std::fclose(f);
      g_err = "bad record framing";
      return 1;
    }
    recs.push_back(std::move(r));
  }
  std::fclose(f);
  const auto sz = rst_sizes(o);
  if (recs.size() < sz.size()) { g_err = "fewer than 49 records"; return 1; }
  for (size_t k = 0; k < sz.size(); ++k)
    if (recs[k].size() != sz[k]) { g_err = "record " + std::to_string(k + 1) + " has the wrong size"; return 1; }
  int32_t dims[9];
  std::memcpy(dims, recs[2].data(), sizeof dims);
  const int32_t want[8] = {o.nx, o.ny, o.nz, o.nzloc - 1, o.nxpp * o.ny, (int32_t)o.ntot, o.nsubd, o.nzloc};
  for (int k = 0; k < 8; ++k)
    if (dims[k] != want[k]) { g_err = "dims differ"; return 1; }
  bool extra = recs.size() > sz.size() && recs[sz.size()].size() == 6 * 4 + 9 * 8;
  int32_t ei[6] = {0, 0, 0, 0, 0, 0};
  double ed[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (extra) {
    std::memcpy(ei, recs[sz.size()].data(), sizeof ei);
    std::memcpy(ed, recs[sz.size()].data() + sizeof ei, sizeof ed);
    extra = ei[0] == 0x32425749 && ei[1] == 1;
  }
  if (mode == 0 && !extra) { g_err = "no continuation record"; return 1; }
  std::memcpy(&o.t, recs[0].data(), 8);                  // restart.f:25
  size_t k = 29;
  for (auto* L : {o.F, o.Fn, o.Fnm, o.Sn, o.Snm})       // restart.f:73-113
    for (int q = 0; q < 4; ++q, ++k) std::memcpy(L[q].data(), recs[k].data(), o.ntot * 8);
  o.ivardt = 0;
  o.idtstep = 0;
  if (mode == 0) {
    o.istep = ei[2];
    o.ivardt = ei[3];
    o.idtstep = ei[4];
    o.istart = ei[5];
    o.dt = ed[0];
    o.cdt = ed[1];
    o.fac1 = ed[2]; o.fac2 = ed[3]; o.fac3 = ed[4];
    o.bdf1 = ed[5]; o.bdf2 = ed[6]; o.bdf3 = ed[7]; o.bdfv = ed[8];
  } else {  // main.f:613-632 with istart = 1
    o.istep = 0;
    o.istart = 1;
    o.cdt = cdtin;
    const double dt1 = o.dt, dt2 = o.cdt * o.dt, dt3 = o.cdt * o.dt;
    o.fac1 = orc_abvar1(dt1, dt2, dt3);
    o.fac2 = orc_abvar2(dt1, dt2, dt3);
    o.fac3 = orc_abvar3(dt1, dt2, dt3);
    o.bdf1 = orc_bdfvar1(dt1, dt2, dt3);
    o.bdf2 = orc_bdfvar2(dt1, dt2, dt3);
    o.bdf3 = orc_bdfvar3(dt1, dt2, dt3);
    o.bdfv = orc_bdfvarv(dt1, dt2, dt3);
  }
  o.fact = 1. / (o.pp.xkappa * o.dt);
  o.facvel = 1. / (o.pp.xnu * o.dt);
  return 0;
}

// output.f:118-265 (plotf): the fields in physical space (horfft +1 on
// copies: the oracle's state is left as it is), after t, the dims and the
// grids; iform 0 unformatted with REAL*4 fields, 1 formatted 5e14.6 / 5i10.
static std::string fortran_e14_6(double v) {
  char out[40];
  if (std::isnan(v)) { std::snprintf(out, sizeof out, "%14s", "NaN"); return out; }
  if (std::isinf(v)) { std::snprintf(out, sizeof out, "%14s", v > 0 ? "Infinity" : "-Infinity"); return out; }
  std::string body = std::signbit(v) ? "-0." : "0.";
  int e = 0;
  if (v != 0.0) {
    char m[40];
    std::snprintf(m, sizeof m, "%.5e", std::fabs(v));  // 6 significant digits
    body += m[0];
    body.append(m + 2, 5);
    e = std::atoi(m + 8) + 1;
  } else {
    body += "000000";
  }
  char ex[16];
  if (std::abs(e) <= 99) std::snprintf(ex, sizeof ex, "E%c%02d", e < 0 ? '-' : '+', std::abs(e));
  else std::snprintf(ex, sizeof ex, "%c%03d", e < 0 ? '-' : '+', std::abs(e));
  body += ex;
  std::snprintf(out, sizeof out, "%14s", body.c_str());
  return out;
}

// one Ew.d cell (w = 14, d = 6) into out (15 bytes)
void orc_format_e14_6(double v, char* out) { std::snprintf(out, 15, "%s", fortran_e14_6(v).c_str()); }

int orc_plotf(void* h, const char* path, int iform) {
  Orc& o = *(Orc*)h;
  std::vector<double> phys[4];
  for (int q = 0; q < 4; ++q) {
    phys[q] = o.F[q];
    horfft(o, phys[q].data(), 1, o.nz);
  }
  FILE* f = std::fopen(path, iform == 0 ? "wb" : "w");
  if (!f) { g_err = std::string("cannot open ") + path; return 1; }
  bool ok = true;
  auto rec = [&](const void* d, uint32_t n) {
    ok = ok && std::fwrite(&n, 4, 1, f) == 1 && (n == 0 || std::fwrite(d, 1, n, f) == n) && std::fwrite(&n, 4, 1, f) == 1;
  };
  if (iform == 0) {
    const int32_t dims[4] = {o.nx, o.ny, o.nz, (int32_t)o.ntot};
    rec(&o.t, 8);
    rec(dims, 16);
    rec(o.xg.data(), 8 * (uint32_t)o.nx);
    rec(o.yg.data(), 8 * (uint32_t)o.ny);
    rec(o.zg.data(), 8 * (uint32_t)o.nz);
    std::vector<float> t4(o.ntot);
    for (int q = 0; q < 4; ++q) {
      for (size_t p = 0; p < o.ntot; ++p) t4[p] = (float)phys[q][p];  // tempout = real(u), output.f:158
      rec(t4.data(), 4 * (uint32_t)o.ntot);
    }
  } else {
    std::string s;
    int col = 0;
    auto put = [&](double v) {
      if (col == 5) { s += '\n'; col = 0; }
      s += fortran_e14_6(v);
      ++col;
    };
    auto endl = [&]() { s += '\n'; col = 0; };
    put(o.t); endl();
    char c[16];
    for (long v : {(long)o.nx, (long)o.ny, (long)o.nz, (long)o.ntot}) { std::snprintf(c, sizeof c, "%10ld", v); s += c; }
    s += '\n';
    for (double v : o.xg) put(v);
    endl();
    for (double v : o.yg) put(v);
    endl();
    for (double v : o.zg) put(v);
    endl();
    for (int q = 0; q < 4; ++q)
      for (double v : phys[q]) put(v);
    endl();
    ok = std::fwrite(s.data(), 1, s.size(), f) == s.size();
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) { g_err = std::string("write error on ") + path; return 1; }
  return 0;
}

void orc_postp(void* h, double* e18, double* w18, double tstart) {
  Orc& o = *(Orc*)h;
  o.tstart = tstart;
  postp(o, e18, w18);
}

void orc_animdump_line(double t, int n, int istep, char* out, int cap) {
  std::snprintf(out, cap, "%s", animdump_line(t, n, istep).c_str());
}

// forcing.f:115-141: rhograd and rhomean(z)
double orc_rhograd(void* h) { return rhograd(*(Orc*)h); }
double orc_rhomean(void* h, double z) { return rhomean(*(Orc*)h, z); }

void orc_set_speclegen(void* h, int n, const char* dir) {
  Orc& o = *(Orc*)h;
  o.nlegspec = n > 0 ? n : 0;
  o.leg_dir = dir ? dir : "";
}

void orc_set_animation(void* h, double dtanim, const char* dir) {
  Orc& o = *(Orc*)h;
  o.dtanim = dtanim > 0 ? dtanim : 0;
  o.anim_dir = dir ? dir : "";
  o.tdump = 0;
  o.ianimc = 0;
}

void orc_step(void* h) { step(*(Orc*)h); }
void orc_run(void* h, int n) {
  for (int s = 0; s < n; ++s) step(*(Orc*)h);
}

// per-step traces of the shipped run's files: probe u(32,1,10), u(32,1,50)
// (uveltest.dat), min/max (minmaxtest.dat), CFL (cfl.dat), averaging counts
void orc_last_maxcalc(void* h, double* probe2, double* mm8, int* mmidx8, double* cfl3, int* cflidx9, int* avg4) {
  Orc* o = (Orc*)h;
  if (probe2) std::memcpy(probe2, o->probe, 2 * 8);
  if (mm8) std::memcpy(mm8, o->mm, 8 * 8);
  if (mmidx8) std::memcpy(mmidx8, o->mm_idx, 8 * 4);
  if (cfl3) std::memcpy(cfl3, o->cfl, 3 * 8);
  if (cflidx9) std::memcpy(cflidx9, o->cfl_idx, 9 * 4);
  if (avg4) std::memcpy(avg4, o->avg_count, 4 * 4);
}
// run maxcalc alone (round trip + diagnostics) on the current state
void orc_maxcalc(void* h) { maxcalc(*(Orc*)h); }

void orc_diag(void* h, double* out3) { diag_energy(*(Orc*)h, out3); }

void orc_horfft(void* h, double* b, int is, int nk) { horfft(*(Orc*)h, b, is, nk); }
void orc_dpdz(void* h, const double* a, double* b) { dpdz(*(Orc*)h, a, b); }
void orc_filter3d(void* h, double* f, int ifourier, int ilegen) {
  filter_3dlegenfourier(*(Orc*)h, f, ifourier, ilegen);
}
void orc_filter_legenpen(void* h, const double* fin, double* fout) { filter_legenpen(*(Orc*)h, fin, fout); }
int orc_interface_avg3d(void* h, double* f) { return interface_avg3d(*(Orc*)h, f); }
void orc_penalty_setup(void* h, double eps) { penalty_setup(*(Orc*)h, *((Orc*)h)->pen0, eps); }
void orc_penalty_main(void* h, double eps, int ifbcbot, int ifbctop, double bcrbot, double bcibot, double bcrtop,
                      double bcitop, double* rhsr, double* rhsi, double* fr, double* fi) {
  BC bc{ifbcbot, ifbctop, bcrbot, bcibot, bcrtop, bcitop};
  penalty_main(*(Orc*)h, *((Orc*)h)->pen0, eps, bc, rhsr, rhsi, fr, fi);
}
// dense assembled matrix (nz x nz column major) for eps and BCs
void orc_penalty_matrix(void* h, double eps, int ifbcbot, int ifbctop, double* a) {
  Orc& o = *(Orc*)h;
  Pen P(o.nsubd);
  penalty_setup(o, P, eps);
  penalty_ends(o, P, eps, ifbcbot, ifbctop);
  std::vector<double> m;
  matrix_assemble(o, P, eps, m);
  std::memcpy(a, m.data(), m.size() * 8);
}
// penalty parameters for eps and BCs: alpha,beta,gamma,delta,tau1,tau2 (nsubd each)
void orc_penalty_params(void* h, double eps, int ifbcbot, int ifbctop, double* out6ns) {
  Orc& o = *(Orc*)h;
  Pen P(o.nsubd);
  penalty_setup(o, P, eps);
  penalty_ends(o, P, eps, ifbcbot, ifbctop);
  int ns = o.nsubd;
  for (int ks = 0; ks < ns; ++ks) {
    out6ns[ks] = P.pa[ks];
    out6ns[ns + ks] = P.pb[ks];
    out6ns[2 * ns + ks] = P.pg[ks];
    out6ns[3 * ns + ks] = P.pd[ks];
    out6ns[4 * ns + ks] = P.pt1[ks];
    out6ns[5 * ns + ks] = P.pt2[ks];
  }
}
// band_lu.f bandlu_solve on a dense matrix
int orc_bandlu_solve(void* h, const double* ain, double* xr, double* xi) {
  Orc& o = *(Orc*)h;
  std::vector<double> a(ain, ain + (size_t)o.nz * o.nz), ab;
  std::vector<int> ipiv;
  int info = band_factor(o, a, ab, ipiv);
  sgbtrs(o.nz, o.nzloc, o.nzloc, ab.data(), 3 * o.nzloc + 1, ipiv.data(), xr);
  sgbtrs(o.nz, o.nzloc, o.nzloc, ab.data(), 3 * o.nzloc + 1, ipiv.data(), xi);
  return info;
}
// band factors (ldab x nz column major) and pivots, for the GPU factor test
int orc_band_factor(void* h, const double* ain, double* ab_out, int* ipiv_out) {
  Orc& o = *(Orc*)h;
  std::vector<double> a(ain, ain + (size_t)o.nz * o.nz), ab;
  std::vector<int> ipiv;
  int info = band_factor(o, a, ab, ipiv);
  std::memcpy(ab_out, ab.data(), ab.size() * 8);
  std::memcpy(ipiv_out, ipiv.data(), ipiv.size() * 4);
  return info;
}

// multistep.f:7-89
double orc_abvar1(double dt1, double dt2, double dt3) {
  double dt123 = 2. * dt1 + 6. * dt2 + 3. * dt3, dt23 = dt2 + dt3;
  return 1. + dt1 * dt123 / (6. * dt2 * dt23);
}
double orc_abvar2(double dt1, double dt2, double dt3) {
  double dt123 = 2. * dt1 + 3. * dt2 + 3. * dt3;
  return -dt1 * dt123 / (6. * dt2 * dt3);
}
double orc_abvar3(double dt1, double dt2, double dt3) {
  double dt12 = 2. * dt1 + 3. * dt2, dt23 = dt2 + dt3;
  return dt1 * dt12 / (6. * dt3 * dt23);
}
double orc_bdfvarv(double dt1, double dt2, double dt3) {
  double dt12 = dt1 + dt2, dt123 = dt1 + dt2 + dt3;
  return 1. + dt1 / dt12 + dt1 / dt123;
}
double orc_bdfvar1(double dt1, double dt2, double dt3) {
  double dt12 = dt1 + dt2, dt23 = dt2 + dt3, dt123 = dt1 + dt2 + dt3;
  double b = -1. - dt1 / dt2 - dt1 / dt123 - dt1 * dt1 / (dt123 * dt2) - dt1 * dt1 * dt12 / (dt123 * dt23 * dt2);
  return -b;
}
double orc_bdfvar2(double dt1, double dt2, double dt3) {
  double dt12 = dt1 + dt2, dt23 = dt2 + dt3, dt123 = dt1 + dt2 + dt3;
  double b = dt1 * dt1 / (dt12 * dt2) + dt1 * dt1 / (dt2 * dt123) + dt1 * dt1 * dt12 / (dt2 * dt23 * dt123) +
             dt1 * dt1 * dt12 / (dt3 * dt23 * dt123);
  return -b;
}
double orc_bdfvar3(double dt1, double dt2, double dt3) {
  double dt12 = dt1 + dt2, dt23 = dt2 + dt3, dt123 = dt1 + dt2 + dt3;
  double b = -dt1 * dt1 * dt12 / (dt3 * dt23 * dt123);
  return -b;
}

}  // extern "C"
