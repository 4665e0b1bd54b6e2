// Drop-in entry points with the reference's names and argument lists, plus
// the remaining handle API (initial condition, diagnostics, isolated solves).
// Included at the end of iw_host.inl.

namespace {

// physical-space copy of a spectral field, with an optional derivative:
// op 0: f, 1: d/dx, 2: d/dy, 3: d/dz.  dst and tmp are device scratch.
template <typename T>
int phys_of(iw_handle* h, FieldSet<T>& fs, const T* src, T* dst, T* tmp, int op) {
  Geo g = geo(h);
  const T* s = src;
  if (op == 3) {
    k_dz_field<T><<<(unsigned)((h->ntot + 255) / 256), 256, 0, h->st>>>(g, src, tmp);
    s = tmp;
  }
  YJobs<T> jb;
  memset(&jb, 0, sizeof jb);
  jb.j[0] = YJob<T>{s, nullptr, dst, op == 2 ? 1 : 0};
  launch_y<T>(h, fs, jb, 1, h->nz, false);
  typedef typename cplx_t<T>::type C;
  const int M = h->nx / 2;
  size_t smem = 2 * (size_t)M * sizeof(C);
  if (op == 1) {
    // multiply by i kx in (kx,y) space
    k_mulikx<T><<<(unsigned)((h->ntot / 2 + 255) / 256), 256, 0, h->st>>>(g, dst);
  }
  k_xfft_field<T><<<h->ny * h->nz, 128, smem, h->st>>>(g, dst, h->nz, 1, h->plx, fs.Wm, fs.Wn);
  CK(cudaGetLastError());
  return 0;
}

template <typename T>
__global__ void k_mean_profiles(Geo g, const T* u, const T* v, const T* w, const T* t, double* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= g.nz) return;
  size_t p = (size_t)k * g.plane;
  out[k] = (double)u[p];
  out[g.nz + k] = (double)v[p];
  out[2 * g.nz + k] = (double)w[p];
  out[3 * g.nz + k] = (double)t[p];
}

template <typename T>
int horfft_dev(iw_handle* h, FieldSet<T>& fs, T* b, int is, int nk) {
  Geo g = geo(h);
  typedef typename cplx_t<T>::type C;
  const int M = h->nx / 2;
  size_t smem = 2 * (size_t)M * sizeof(C);
  YJobs<T> jb;
  memset(&jb, 0, sizeof jb);
  if (is == -1) {
    k_xfft_field<T><<<h->ny * nk, 128, smem, h->st>>>(g, b, nk, 0, h->plx, fs.Wm, fs.Wn);
    jb.j[0] = YJob<T>{b, nullptr, b, 2};
    launch_y<T>(h, fs, jb, 1, nk, false);
  } else {
    jb.j[0] = YJob<T>{b, nullptr, b, 0};
    launch_y<T>(h, fs, jb, 1, nk, false);
    k_xfft_field<T><<<h->ny * nk, 128, smem, h->st>>>(g, b, nk, 1, h->plx, fs.Wm, fs.Wn);
  }
  CK(cudaGetLastError());
  return 0;
}

uint64_t xs_next(uint64_t& s) {
  s ^= s << 21;
  s ^= s >> 35;
  s ^= s << 4;
  return s;
}

// per-call device scratch of n doubles
struct DBuf {
  double* p = nullptr;
  explicit DBuf(size_t n) { cudaMalloc(&p, n * sizeof(double) + 16); }
  ~DBuf() { cudaFree(p); }
};

iw_handle* bound() {
  if (!g_bound) set_err(IW_ERR_STATE, "no handle bound (iw_bind)");
  return g_bound;
}

double g_setup_eps = -1.0;

// one penalty system for eps and BCs, assembled, factored (1 warp), and
// used to solve for nr right-hand sides b[r*nz + k] (device).
__global__ void k_solve_one(Geo g, const double* ab, const int* ipiv, double* b, int nr) {
  extern __shared__ double sb[];
  const int n = g.nz;
  for (int t = threadIdx.x; t < nr * n; t += 32) sb[t] = b[t];
  __syncwarp();
  band_solve_warp(ab, ipiv, sb, nr, n, g.N, g.N, threadIdx.x);
  for (int t = threadIdx.x; t < nr * n; t += 32) b[t] = sb[t];
}

__global__ void k_legen_one(Geo g, const double* wg, const double* alpol, const double* sigma, double* b, int N) {
  legen_filter_cols(b, 1, N, N, 1, wg, alpol, sigma, threadIdx.x);
}

int factor_dense_or_params(iw_handle* h, const double* pen6, double eps, int bot, int top, const double* dense,
                           double** ab_out, int** ipiv_out) {
  const int n = h->nz, N = h->N, ldab = 3 * N + 1, ns = h->ns;
  g_status = 0;
  SysDesc sd;
  memset(&sd, 0, sizeof sd);
  sd.eps = eps;
  sd.ifbcbot = bot;
  sd.ifbctop = top;
  SysDesc* dsd;
  double *dpen, *dab;
  int *dip, *dinfo;
  CK(cudaMalloc(&dsd, sizeof sd));
  CK(cudaMalloc(&dpen, 6 * ns * sizeof(double)));
  CK(cudaMalloc(&dab, (size_t)ldab * n * sizeof(double)));
  CK(cudaMalloc(&dip, n * sizeof(int)));
  CK(cudaMalloc(&dinfo, sizeof(int)));
  CK(scopy(h, dsd, &sd, sizeof sd, cudaMemcpyHostToDevice));
  CK(scopy(h, dpen, pen6, 6 * ns * sizeof(double), cudaMemcpyHostToDevice));
  FactorArgs fa;
  fa.sys = dsd;
  fa.pen = dpen;
  fa.ab = dab;
  fa.ipiv = dip;
  fa.info = dinfo;
  fa.nsys = 1;
  fa.D = h->dD;
  fa.D2 = h->dD2;
  fa.zh = h->dzh;
  fa.assemble = 1;
  if (dense) {
    // band_lu.f:19-34 packing done on the host
    std::vector<double> ab((size_t)ldab * n, 0.0);
    for (int j = 1; j <= n; ++j)
      for (int i = std::max(1, j - N); i <= std::min(n, j + N); ++i)
        ab[(size_t)(2 * N + i - j) + (size_t)ldab * (j - 1)] = dense[(size_t)(i - 1) + (size_t)n * (j - 1)];
    CK(scopy(h, dab, ab.data(), ab.size() * sizeof(double), cudaMemcpyHostToDevice));
    fa.assemble = 0;
  }
  k_factor<<<1, 32, 0, h->st>>>(geo(h), fa);
  int info = 0;
  CK(scopy(h, &info, dinfo, sizeof info, cudaMemcpyDeviceToHost));
  cudaFree(dsd);
  cudaFree(dpen);
  cudaFree(dinfo);
  // SGBTF2's INFO (bandludcmp.f:238-440): the reference ignores it (band_lu.f:23-34)
  // and so does the solve that follows; it is recorded for iw_last_status.
  if (info > 0) set_err(IW_ERR_PIVOT, "zero pivot in band factorisation at column " + std::to_string(info));
  *ab_out = dab;
  *ipiv_out = dip;
  return 0;
}

}  // namespace

// ---------------------------------------------------------------------------
// K_A..K_E and the solves as the reference's two calls
// ---------------------------------------------------------------------------
extern "C" {

void convec_(const int* istep, const int* istart, const int* ispecfilternl) {
  iw_handle* h = bound();
  if (!h) return;
  (void)istart;
  int save = h->p.ispecfilternl;
  if (ispecfilternl) h->p.ispecfilternl = *ispecfilternl;
  if (istep) h->istep = *istep;
  if (h->mixed)
    convec_impl<float>(h, h->f32, 0);
  else
    convec_impl<double>(h, h->f64, 0);
  h->p.ispecfilternl = save;
}

void calcuvwt_(const int* izmode, const int* ispecfilter, const int* irelax, const int* cpenspecfilter) {
  (void)izmode;
  (void)ispecfilter;
  (void)irelax;
  iw_handle* h = bound();
  if (!h) return;
  int cpen = cpenspecfilter ? (*cpenspecfilter != 0) : 1;
  if (ensure_factors(h, cpen)) return;
  if (h->mixed)
    calcuvwt_impl<float>(h, h->f32, cpen);
  else
    calcuvwt_impl<double>(h, h->f64, cpen);
}

void horfft_(double* b, const int* is, const int* nk) {
  iw_handle* h = bound();
  if (!h || !b || !is || !nk) return;
  size_t n = h->plane * (size_t)*nk;
  DBuf d(n);
  scopy(h, d.p, b, n * sizeof(double), cudaMemcpyHostToDevice);
  FieldSet<double> tmp;
  typedef double2 C;
  int M = h->nx / 2;
  auto wm = twiddles<C>(M, M);
  auto wn = twiddles<C>(h->nx, M + 1);
  auto wy = twiddles<C>(h->ny, h->ny);
  if (up(h, &tmp.Wm, wm) || up(h, &tmp.Wn, wn) || up(h, &tmp.Wy, wy)) return;
  horfft_dev<double>(h, tmp, d.p, *is, *nk);
  cudaStreamSynchronize(h->st);
  scopy(h, b, d.p, n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(tmp.Wm);
  cudaFree(tmp.Wn);
  cudaFree(tmp.Wy);
}

void dpdz_(const double* a, double* b) {
  iw_handle* h = bound();
  if (!h || !a || !b) return;
  DBuf da(h->ntot), db(h->ntot);
  scopy(h, da.p, a, h->ntot * sizeof(double), cudaMemcpyHostToDevice);
  k_dz_field<double><<<(unsigned)((h->ntot + 255) / 256), 256, 0, h->st>>>(geo(h), da.p, db.p);
  cudaStreamSynchronize(h->st);
  scopy(h, b, db.p, h->ntot * sizeof(double), cudaMemcpyDeviceToHost);
}

void filter_3dlegenfourier_(double* f, const int* ifourier, const int* ilegen, const int* iout) {
  (void)iout;
  iw_handle* h = bound();
  if (!h || !f) return;
  DBuf d(h->ntot);
  scopy(h, d.p, f, h->ntot * sizeof(double), cudaMemcpyHostToDevice);
  long total = (long)h->nxpp * h->ny * h->ns;
  k_filter_field<double><<<(unsigned)((total + 127) / 128), 128, 0, h->st>>>(geo(h), d.p, ifourier ? *ifourier : 1,
                                                                            ilegen ? *ilegen : 1);
  cudaStreamSynchronize(h->st);
  scopy(h, f, d.p, h->ntot * sizeof(double), cudaMemcpyDeviceToHost);
}

void filter_legenpen_(const double* fin, double* fout, const double* ybar, const int* iprt, const int* ks) {
  (void)ybar;
  (void)iprt;
  (void)ks;
  iw_handle* h = bound();
  if (!h || !fin || !fout) return;
  DBuf d(h->N);
  scopy(h, d.p, fin, h->N * sizeof(double), cudaMemcpyHostToDevice);
  k_legen_one<<<1, 32, 0, h->st>>>(geo(h), h->dwg, h->dal, h->dsig, d.p, h->N);
  cudaStreamSynchronize(h->st);
  scopy(h, fout, d.p, h->N * sizeof(double), cudaMemcpyDeviceToHost);
}

void interface_avg3d_(double* f, int* ic) {
  iw_handle* h = bound();
  if (!h || !f) return;
  FieldSet<double> fs;
  DBuf d(h->ntot), G(h->plane * 16 * (size_t)std::max(1, h->ns - 1));
  typedef double2 C;
  int M = h->nx / 2;
  auto wm = twiddles<C>(M, M);
  auto wn = twiddles<C>(h->nx, M + 1);
  auto wy = twiddles<C>(h->ny, h->ny);
  if (up(h, &fs.Wm, wm) || up(h, &fs.Wn, wn) || up(h, &fs.Wy, wy)) return;
  scopy(h, d.p, f, h->ntot * sizeof(double), cudaMemcpyHostToDevice);
  for (int q = 0; q < 4; ++q) fs.F[q] = d.p;
  fs.G = G.p;
  iface_avg<double>(h, fs, true, 1);
  cudaStreamSynchronize(h->st);
  scopy(h, f, d.p, h->ntot * sizeof(double), cudaMemcpyDeviceToHost);
  if (ic) {
    int cnt[4];
    scopy(h, cnt, h->dcnt, sizeof cnt, cudaMemcpyDeviceToHost);
    *ic = cnt[0];
  }
  fs.F[0] = fs.F[1] = fs.F[2] = fs.F[3] = nullptr;
  fs.G = nullptr;
  cudaFree(fs.Wm);
  cudaFree(fs.Wn);
  cudaFree(fs.Wy);
  fs.Wm = fs.Wn = fs.Wy = nullptr;
}

void penalty_setup_(const double* epsilon) {
  if (epsilon) g_setup_eps = *epsilon;
}

void penalty_main_(const double* epsilon, const int* ifuncreal, const double* bcrbot, const double* bcibot,
                   const double* bcrtop, const double* bcitop, const int* ifbcbot, const int* ifbctop, double* rhsinr,
                   double* rhsini, double* fr, double* fi) {
  (void)ifuncreal;
  iw_handle* h = bound();
  if (!h) return;
  const int n = h->nz, ns = h->ns;
  const double eps = *epsilon;
  std::vector<double> pen(6 * ns), pen_int(6 * ns);
  h_penalty(ns, h->N, h->p, eps, *ifbcbot, *ifbctop, pen.data());
  if (g_setup_eps > 0 && g_setup_eps != eps) {
    // interior subdomains keep the parameters of the last penalty_setup
    h_penalty(ns, h->N, h->p, g_setup_eps, *ifbcbot, *ifbctop, pen_int.data());
    for (int a = 0; a < 6; ++a)
      for (int ks = 1; ks < ns - 1; ++ks) pen[a * ns + ks] = pen_int[a * ns + ks];
  }
  for (int k = 0; k < n; ++k) {
    rhsinr[k] = -(rhsinr[k] * eps);
    rhsini[k] = -(rhsini[k] * eps);
  }
  std::vector<double> b(2 * (size_t)n);
  for (int k = 0; k < n; ++k) {
    b[k] = rhsinr[k];
    b[n + k] = rhsini[k];
  }
  const double t1 = pen[4 * ns + 0], t2 = pen[5 * ns + ns - 1];
  if (*ifbcbot == 0) {
    b[0] = rhsinr[0] + t1 * *bcrbot;
    b[n] = rhsini[0] + t1 * *bcibot;
  } else {
    b[0] = rhsinr[0] - t1 * *bcrbot * eps;
    b[n] = rhsini[0] - t1 * *bcibot * eps;
  }
  if (*ifbctop == 0) {
    b[n - 1] = rhsinr[n - 1] + t2 * *bcrtop;
    b[2 * n - 1] = rhsini[n - 1] + t2 * *bcitop;
  } else {
    b[n - 1] = rhsinr[n - 1] + t2 * *bcrtop * eps;
    b[2 * n - 1] = rhsini[n - 1] + t2 * *bcitop * eps;
  }
  double* dab;
  int* dip;
  if (factor_dense_or_params(h, pen.data(), eps, *ifbcbot, *ifbctop, nullptr, &dab, &dip)) return;
  DBuf db(2 * (size_t)n);
  scopy(h, db.p, b.data(), b.size() * sizeof(double), cudaMemcpyHostToDevice);
  k_solve_one<<<1, 32, 2 * n * sizeof(double), h->st>>>(geo(h), dab, dip, db.p, 2);
  cudaStreamSynchronize(h->st);
  scopy(h, b.data(), db.p, b.size() * sizeof(double), cudaMemcpyDeviceToHost);
  for (int k = 0; k < n; ++k) {
    fr[k] = b[k];
    fi[k] = b[n + k];
  }
  cudaFree(dab);
  cudaFree(dip);
}

void bandlu_solve_(const double* ain, double* xr, double* xi, const int* ifuncreal) {
  iw_handle* h = bound();
  if (!h) return;
  const int n = h->nz;
  std::vector<double> pen(6 * h->ns, 0.0);
  double* dab;
  int* dip;
  if (factor_dense_or_params(h, pen.data(), 1.0, 0, 0, ain, &dab, &dip)) return;
  int nr = (ifuncreal && *ifuncreal == 1) ? 1 : 2;
  std::vector<double> b(2 * (size_t)n);
  for (int k = 0; k < n; ++k) {
    b[k] = xr[k];
    b[n + k] = xi ? xi[k] : 0.0;
  }
  DBuf db(2 * (size_t)n);
  scopy(h, db.p, b.data(), b.size() * sizeof(double), cudaMemcpyHostToDevice);
  k_solve_one<<<1, 32, 2 * n * sizeof(double), h->st>>>(geo(h), dab, dip, db.p, nr);
  cudaStreamSynchronize(h->st);
  scopy(h, b.data(), db.p, b.size() * sizeof(double), cudaMemcpyDeviceToHost);
  for (int k = 0; k < n; ++k) {
    xr[k] = b[k];
    if (xi && nr == 2) xi[k] = b[n + k];
  }
  cudaFree(dab);
  cudaFree(dip);
}

// multistep.f:7-89
double abvar1_(const double* a, const double* b, const double* c) {
  double dt1 = *a, dt2 = *b, dt3 = *c;
  double dt123 = 2. * dt1 + 6. * dt2 + 3. * dt3, dt23 = dt2 + dt3;
  return 1. + dt1 * dt123 / (6. * dt2 * dt23);
}
double abvar2_(const double* a, const double* b, const double* c) {
  double dt1 = *a, dt2 = *b, dt3 = *c;
  double dt123 = 2. * dt1 + 3. * dt2 + 3. * dt3;
  return -dt1 * dt123 / (6. * dt2 * dt3);
}
double abvar3_(const double* a, const double* b, const double* c) {
  double dt1 = *a, dt2 = *b, dt3 = *c;
  double dt12 = 2. * dt1 + 3. * dt2, dt23 = dt2 + dt3;
  return dt1 * dt12 / (6. * dt3 * dt23);
}
double bdfvarv_(const double* a, const double* b, const double* c) {
  double dt1 = *a, dt2 = *b, dt3 = *c;
  double dt12 = dt1 + dt2, dt123 = dt1 + dt2 + dt3;
  return 1. + dt1 / dt12 + dt1 / dt123;
}
double bdfvar1_(const double* a, const double* b, const double* c) {
  double dt1 = *a, dt2 = *b, dt3 = *c;
  double dt12 = dt1 + dt2, dt23 = dt2 + dt3, dt123 = dt1 + dt2 + dt3;
  double r = -1. - dt1 / dt2 - dt1 / dt123 - dt1 * dt1 / (dt123 * dt2) - dt1 * dt1 * dt12 / (dt123 * dt23 * dt2);
  return -r;
}
double bdfvar2_(const double* a, const double* b, const double* c) {
  double dt1 = *a, dt2 = *b, dt3 = *c;
  double dt12 = dt1 + dt2, dt23 = dt2 + dt3, dt123 = dt1 + dt2 + dt3;
  double r = dt1 * dt1 / (dt12 * dt2) + dt1 * dt1 / (dt2 * dt123) + dt1 * dt1 * dt12 / (dt2 * dt23 * dt123) +
             dt1 * dt1 * dt12 / (dt3 * dt23 * dt123);
  return -r;
}
double bdfvar3_(const double* a, const double* b, const double* c) {
  double dt1 = *a, dt2 = *b, dt3 = *c;
  double dt12 = dt1 + dt2, dt23 = dt2 + dt3, dt123 = dt1 + dt2 + dt3;
  double r = -dt1 * dt1 * dt12 / (dt3 * dt23 * dt123);
  return -r;
}

// ---------------------------------------------------------------------------
int iw_init_mode1(iw_handle* h, double A, double anoise, uint64_t seed) {
  if (!h) return set_err(IW_ERR_STATE, "null handle");
  cudaSetDevice(h->dev);
  const int nx = h->nx, ny = h->ny, nz = h->nz, nxpp = h->nxpp;
  const double pi2 = 8. * std::atan(1.0);
  const double kx = pi2 / h->p.xlen, m = pi2 / (2. * h->p.zlen);
  const double om = (h->p.brunt * kx) / std::sqrt(kx * kx + m * m);
  const double rc = (h->p.rho0 * h->p.brunt * h->p.brunt) / h->p.grav;
  const double xl = pi2 / (pi2 / h->p.xlen);
  std::vector<double> zg(nz);
  for (int ks = 0; ks < h->ns; ++ks)
    for (int kl = 0; kl < h->N; ++kl) zg[ks * h->N + kl] = h->p.z0[ks] + 0.5 * h->p.zh[ks] * (h->tab.zpts[kl] + 1.0);
  std::vector<double> st(4 * h->ntot, 0.0);
  auto at = [&](int q, int i, int j, int k) -> double& {
    return st[(size_t)q * h->ntot + (size_t)i + (size_t)nxpp * ((size_t)j + (size_t)ny * k)];
  };
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        double x = i * xl / nx, z = zg[k];
        at(0, i, j, k) = -(A / kx) * m * std::cos(m * z) * std::sin(kx * x);
        at(2, i, j, k) = A * std::sin(m * z) * std::cos(kx * x);
        at(3, i, j, k) = -(A / om) * rc * std::sin(m * z) * std::sin(kx * x);
      }
  uint64_t s = seed ? seed : 0x9E3779B97F4A7C15ULL;
  for (int k = 0; k < nz; ++k) {
    if (!(zg[k] < 0.2 * h->p.zlen)) continue;
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        for (int q = 0; q < 3; ++q) {
          uint64_t v = xs_next(s);
          double r = (double)(int64_t)v * 5.42101086242752217e-20 + 0.5;
          at(q, i, j, k) += anoise * (2.0 * r - 1.0);
        }
  }
  std::vector<double> zero(4 * h->ntot, 0.0);
  int r = iw_upload_state(h, h->mixed ? nullptr : st.data(), zero.data(), zero.data(), zero.data(), zero.data(), 0.0, 0);
  if (r) return r;
  if (h->mixed) {
    // The forward transform of the initial fields runs in FP64 and only the
    // spectral result is rounded to FP32, coefficient by coefficient.  An FP32
    // transform would spread its rounding (relative to the wave's amplitude)
    // over every (kx, ky) mode of u and w, and the first projection would
    // carry that divergent noise into v, a field about 1000 times smaller.
    FieldSet<double> tmp;
    typedef double2 C;
    const int M = nx / 2;
    auto wm = twiddles<C>(M, M);
    auto wn = twiddles<C>(nx, M + 1);
    auto wy = twiddles<C>(ny, ny);
    if (up(h, &tmp.Wm, wm) || up(h, &tmp.Wn, wn) || up(h, &tmp.Wy, wy)) return IW_ERR_NOMEM;
    DBuf d(h->ntot);
    if (!d.p) return set_err(IW_ERR_NOMEM, "iw_init_mode1: no memory for the FP64 transform");
    for (int q = 0; q < 4 && r == 0; ++q) {
      if (cudaMemcpyAsync(d.p, st.data() + (size_t)q * h->ntot, h->ntot * sizeof(double), cudaMemcpyHostToDevice,
                          h->st) != cudaSuccess) {
        r = set_err(IW_ERR_CUDA, "iw_init_mode1: copy of the initial field");
        break;
      }
      horfft_dev<double>(h, tmp, d.p, -1, nz);
      k_convert<double, float><<<1184, 256, 0, h->st>>>(d.p, h->f32.F[q], h->ntot);
    }
    cudaStreamSynchronize(h->st);
    cudaFree(tmp.Wm);
    cudaFree(tmp.Wn);
    cudaFree(tmp.Wy);
    if (r) return r;
  } else {
    for (int q = 0; q < 4; ++q) horfft_dev<double>(h, h->f64, h->f64.F[q], -1, nz);
  }
  CK(cudaMemsetAsync(h->dwnl, 0, h->plane * 2 * sizeof(double), h->st));
  CK(cudaMemsetAsync(h->dwvr, 0, h->plane * 2 * sizeof(double), h->st));
  CK(cudaStreamSynchronize(h->st));
  return IW_OK;
}

}  // extern "C"

template <typename T>
static int diag_impl(iw_handle* h, FieldSet<T>& fs, iw_diag_out* out) {
  Geo g = geo(h);
  T* dst = fs.Y12[0];
  T* tmp = fs.Y12[1];
  // KE: u,v,w ; eps: 9 gradients.  Per-block slots (296 for KE, 296 for
  // eps) in the second half of dpart, added in order on the host.
  double* rp = h->dpart + (size_t)4 * 296 * 5;
  CK(cudaMemsetAsync(rp, 0, 2 * 296 * sizeof(double), h->st));
  for (int q = 0; q < 3; ++q) {
    phys_of<T>(h, fs, fs.F[q], dst, tmp, 0);
    k_reduce_sq<T><<<296, 256, 0, h->st>>>(g, dst, 1, rp);
    for (int op = 1; op <= 3; ++op) {
      phys_of<T>(h, fs, fs.F[q], dst, tmp, op);
      k_reduce_sq<T><<<296, 256, 0, h->st>>>(g, dst, 1, rp + 296);
    }
  }
  double red[2] = {0, 0};
  // maxcalc statistics on the physical fields
  {
    const double dx = h->p.xlen / h->nx, dy = h->p.ylen / h->ny;
    const double rg = -(h->p.rho0 * h->p.brunt * h->p.brunt) / h->p.grav;
    for (int q = 0; q < 4; ++q) {
      phys_of<T>(h, fs, fs.F[q], dst, tmp, 0);
      const double cflh = q == 0 ? h->p.dt / dx : q == 1 ? h->p.dt / dy : 0.0;
      k_phys_stats<T><<<296, 256, 0, h->st>>>(g, dst, q, h->dzg, h->ddzinv, cflh, rg, 0.2 * h->p.zlen,
                                              h->dpart + (size_t)q * 296 * 5);
    }
  }
  std::vector<double> part((size_t)4 * 296 * 5 + 2 * 296);
  CK(cudaMemcpyAsync(part.data(), h->dpart, part.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  for (int b = 0; b < 296; ++b) {
    red[0] += part[(size_t)4 * 296 * 5 + b];
    red[1] += part[(size_t)4 * 296 * 5 + 296 + b];
  }
  memset(out, 0, sizeof *out);
  {
    double mm[4][2], cf[4] = {0, 0, 0, 0}, s2 = 0, cnt = 0;
    for (int q = 0; q < 4; ++q) {
      mm[q][0] = part[(size_t)q * 296 * 5];
      mm[q][1] = part[(size_t)q * 296 * 5 + 1];
      for (int b = 0; b < 296; ++b) {
        const double* o = part.data() + ((size_t)q * 296 + b) * 5;
        mm[q][0] = std::min(mm[q][0], o[0]);
        mm[q][1] = std::max(mm[q][1], o[1]);
        cf[q] = std::max(cf[q], o[2]);
        if (q == 2) {
          s2 += o[3];
          cnt += o[4];
        }
      }
    }
    out->umin = mm[0][0];
    out->umax = mm[0][1];
    out->vmin = mm[1][0];
    out->vmax = mm[1][1];
    out->wmin = mm[2][0];
    out->wmax = mm[2][1];
    out->tmin = mm[3][0];
    out->tmax = mm[3][1];
    out->cflx = cf[0];
    out->cfly = cf[1];
    out->cflz = cf[2];
    out->wrms_bottom = cnt > 0 ? std::sqrt(s2 / cnt) : 0.0;
  }
  out->ke = 0.5 * red[0];
  out->eps = h->p.xnu * red[1];
  out->t = h->t;
  out->dt = h->p.dt;
  out->istep = h->istep;
  int cnt[4] = {0, 0, 0, 0};
  CK(scopy(h, cnt, h->dcnt, sizeof cnt, cudaMemcpyDeviceToHost));
  for (int q = 0; q < 4; ++q) out->interface_avg_count[q] = cnt[q];
  // non-finite check of the state
  CK(cudaMemsetAsync(h->dflag, 0, sizeof(int), h->st));
  for (int q = 0; q < 4; ++q) k_nonfinite<T><<<296, 256, 0, h->st>>>(fs.F[q], h->ntot, h->dflag);
  int flag = 0;
  CK(cudaMemcpyAsync(&flag, h->dflag, sizeof flag, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  if (flag) return set_err(IW_ERR_NONFINITE, "non-finite value in the state");
  return sync_errors(h);
}

// CFL numbers of the state for the adaptive rule: maxcalc's cflxmax and
// cflzmax (various.f:780-870), from the same per-block partials as iw_diag.
template <typename T>
static int step_cfl(iw_handle* h, FieldSet<T>& fs, double* cflx, double* cflz) {
  Geo g = geo(h);
  T* dst = fs.Y12[0];
  T* tmp = fs.Y12[1];
  const double dx = h->p.xlen / h->nx, rg = -(h->p.rho0 * h->p.brunt * h->p.brunt) / h->p.grav;
  for (int q = 0; q <= 2; q += 2) {
    phys_of<T>(h, fs, fs.F[q], dst, tmp, 0);
    k_phys_stats<T><<<296, 256, 0, h->st>>>(g, dst, q, h->dzg, h->ddzinv, q == 0 ? h->p.dt / dx : 0.0, rg,
                                            0.2 * h->p.zlen, h->dpart + (size_t)q * 296 * 5);
  }
  std::vector<double> part((size_t)3 * 296 * 5);
  CK(cudaMemcpyAsync(part.data(), h->dpart, part.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  double cf[2] = {0, 0};
  for (int b = 0; b < 296; ++b) {
    cf[0] = std::max(cf[0], part[(size_t)b * 5 + 2]);
    cf[1] = std::max(cf[1], part[((size_t)2 * 296 + b) * 5 + 2]);
  }
  *cflx = cf[0];
  *cflz = cf[1];
  return IW_OK;
}

extern "C" {

// various.f:892-982; the step count is taken from t = 0 (see the header)
int iw_dt_rule(double cflx, double cflz, double t, double dt, double xomega, double* dt_new, double* cdt) {
  if (!(dt > 0) || !dt_new || !cdt) return 0;
  const bool change_dt = cflz > 0.7 || cflz < 0.1 || cflx > 0.16;
  const double pi2 = 8. * std::atan(1.0);
  const double tlim = pi2 / (xomega * 50.);
  if (!(std::trunc(t / dt) > 20.0) || !change_dt) return 0;
  double c = 1.;
  if (cflz < 0.1) c = std::max(0.8, dt / tlim);
  if (cflz > 0.7 || cflx > 0.16) c = 1.25;
  *cdt = c;
  *dt_new = dt / c;
  return 1;
}

int iw_diag(iw_handle* h, iw_diag_out* out) {
  if (!h || !out) return set_err(IW_ERR_STATE, "bad argument");
  cudaSetDevice(h->dev);
  return h->mixed ? diag_impl<float>(h, h->f32, out) : diag_impl<double>(h, h->f64, out);
}

// Mean (kx=ky=0) vertical profiles of u,v,w,rho copied to the host: the
// per-step result a driver reads back.
int iw_mean_profiles(iw_handle* h, double* host4nz) {
  if (!h || !host4nz) return set_err(IW_ERR_STATE, "bad argument");
  cudaSetDevice(h->dev);
  Geo g = geo(h);
  unsigned nb = (unsigned)((h->nz + 127) / 128);
  if (h->mixed)
    k_mean_profiles<float><<<nb, 128, 0, h->st>>>(g, h->f32.F[0], h->f32.F[1], h->f32.F[2], h->f32.F[3], h->dred);
  else
    k_mean_profiles<double><<<nb, 128, 0, h->st>>>(g, h->f64.F[0], h->f64.F[1], h->f64.F[2], h->f64.F[3], h->dred);
  CK(cudaMemcpyAsync(host4nz, h->dred, 4 * (size_t)h->nz * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return IW_OK;
}

// Isolated batched solves: one system per column with lambda = lam[c].
int iw_helm_solve_batched(iw_handle* h, const double* lam_dev, int ncol, int ifbcbot, int ifbctop,
                          const double* rhs_dev, double* sol_dev, int mode) {
  if (!h || !lam_dev || !rhs_dev || !sol_dev || ncol <= 0) return set_err(IW_ERR_STATE, "bad argument");
  cudaSetDevice(h->dev);
  return helm_batched(h, lam_dev, ncol, ifbcbot, ifbctop, rhs_dev, sol_dev, mode);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// bandlu_solve_ without device allocation.
//
// Some callers cannot allocate device memory while they run. Examples: a
// program whose device memory is handed out by its own pool, sized at start-up
// (a fresh cudaMalloc may fail or is not allowed), or a timing-critical loop
// that cannot take the device-wide synchronisation implied by cudaFree.
// iw_bandlu_solve_noalloc does the work of bandlu_solve_ (pack the dense matrix
// into band storage, factor with partial pivoting, solve in place) with the
// same kernels.  Its band storage, pivots and status live in one fixed
// file-scope device array of kNoAllocDoubles doubles (about 1.06 MB), which
// every GPU that loads this library keeps until the process exits.
// ---------------------------------------------------------------------------
namespace {
constexpr size_t kNoAllocBand = 131072;  // band storage: (3 nzloc + 1) * nz doubles at most
// nz bound of the pivot storage and of the solve's shared memory (two right-hand
// sides stay within 48 KB); the band bound above is the tighter one: with
// nzloc, nsubd <= 64 it allows nz <= 1600
constexpr int kNoAllocMaxN = 3072;
constexpr size_t kNoAllocPivot = kNoAllocBand;                  // pivots: kNoAllocMaxN ints
constexpr size_t kNoAllocInfo = kNoAllocPivot + kNoAllocMaxN / 2;  // status word
constexpr size_t kNoAllocSys = kNoAllocInfo + 8;               // system descriptor
constexpr size_t kNoAllocDoubles = kNoAllocSys + 56;
static_assert(sizeof(SysDesc) <= 56 * sizeof(double), "SysDesc must fit its scratch slot");
constexpr int kNoAllocMaxDev = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_base[kNoAllocMaxDev] = {};
}  // namespace

// Shared by every call on a device; see iw_bandlu_solve_noalloc for the rules.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

// Column-major dense n x n -> band storage of band_lu.f:19-34 (row 2N + i - j
// of column j holds a(i, j) for |i - j| <= N).  Every entry is written, the N
// fill-in rows and everything outside the band as zero, so nothing left by an
// earlier call survives.  Also resets the status word and the descriptor.
__global__ void k_pack_band(const double* __restrict__ a, int n, int N, int ldab, double* __restrict__ ab,
                            SysDesc* sd, int* info) {
  const size_t tot = (size_t)ldab * n;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < tot; q += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(q % ldab), j = (int)(q / ldab);
    const int i = r - 2 * N + j;
    ab[q] = (r >= N && i >= 0 && i < n) ? a[(size_t)i + (size_t)n * j] : 0.0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    SysDesc s;
    memset(&s, 0, sizeof s);
    s.eps = 1.0;
    *sd = s;
    *info = 0;
  }
}

extern "C" {

int iw_bandlu_solve_noalloc(const double* ain_dev, double* x_dev, int nzloc, int nsubd, int nrhs, void* stream) {
  if (!ain_dev || !x_dev) return set_err(IW_ERR_STATE, "iw_bandlu_solve_noalloc: null matrix or right-hand side");
  if (nzloc < 2 || nsubd < 1 || nzloc > IW_MAX_NZLOC || nsubd > IW_MAX_SUBD)
    return set_err(IW_ERR_CONFIG, "iw_bandlu_solve_noalloc: nzloc must be in [2, 64] and nsubd in [1, 64]");
  if (nrhs != 1 && nrhs != 2) return set_err(IW_ERR_CONFIG, "iw_bandlu_solve_noalloc: nrhs must be 1 or 2");
  const int n = nzloc * nsubd, ldab = 3 * nzloc + 1;
  if (n > kNoAllocMaxN || (size_t)ldab * n > kNoAllocBand)
    return set_err(IW_ERR_CONFIG, "iw_bandlu_solve_noalloc: system exceeds the fixed scratch: need "
                                  "(3*nzloc+1)*nzloc*nsubd <= 131072, got nz=" +
                                      std::to_string(n) + ", band " + std::to_string((size_t)ldab * n));
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDev) return set_err(IW_ERR_CONFIG, "iw_bandlu_solve_noalloc: device index too large");
  double* base = nullptr;
  {
    // one-time set-up per device, with that device current: the device
    // address of the scratch array (its name in host code is not one)
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_base[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p)
        return set_err(IW_ERR_CUDA, std::string("iw_bandlu_solve_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_noalloc_base[dev] = (double*)p;
    }
    base = g_noalloc_base[dev];
  }
  double* ab = base;
  int* ipiv = (int*)(base + kNoAllocPivot);
  int* info = (int*)(base + kNoAllocInfo);
  SysDesc* sd = (SysDesc*)(base + kNoAllocSys);
  Geo g;
  memset(&g, 0, sizeof g);
  g.nz = n;
  g.N = nzloc;
  g.ns = nsubd;
  FactorArgs fa;
  memset(&fa, 0, sizeof fa);
  fa.sys = sd;
  fa.pen = base;  // not read without assembly
  fa.ab = ab;
  fa.ipiv = ipiv;
  fa.info = info;
  fa.nsys = 1;
  fa.assemble = 0;
  fa.factor = 1;
  cudaStream_t st = (cudaStream_t)stream;
  k_pack_band<<<64, 256, 0, st>>>(ain_dev, n, nzloc, ldab, ab, sd, info);
  k_factor<<<1, 32, 0, st>>>(g, fa);
  k_solve_one<<<1, 32, (size_t)nrhs * n * sizeof(double), st>>>(g, ab, ipiv, x_dev, nrhs);
  CK(cudaGetLastError());
  return IW_OK;
}

}  // extern "C"
