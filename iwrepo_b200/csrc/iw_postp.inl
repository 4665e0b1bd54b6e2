// TKE budget: postp.f:9-70 (postp) with umeancalc (postp.f:129-213),
// dudzmeancalc / dpdzyzplane (postp.f:215-235, 984-1020), dudymeancalc
// (postp.f:237-298), perturbcalc (postp.f:300-330) and energycalc_postp
// (postp.f:415-732).
//
// In physical space: umean(j,k) is the x mean of u for k >= 2 and 0 at k = 1;
// u' = u - umean; u', v, w and temp are transformed to spectral space, their
// gradients taken there (i kx, i ky, the subdomain z derivative), and all are
// transformed back before the sums, as energycalc_postp does.  Over k = 2..nz,
// all j and i = 1..nx:
//   tketot = 1/2 sum (u'^2 + v^2 + w^2), u1tke = sum u'^2, u2tke, u3tke,
//   prody = -sum dumeandy u' v, prodz = -sum dumeandz u' w, prod = prody + prodz,
//   bflux = ra pr sum w temp (ra = 0: the reference's start-up value),
//   epsilon = pr sum |grad(u', v, w)|^2 (pr = xnu), chi = xkappa sum |grad temp|^2,
//   tkemean = nx/2 sum_{j,k} umean^2, tempvar = sum temp^2.
// The subgrid terms epssgs and chisgs are 0 (no subgrid model: t11... and
// th1... stay 0), so epstot = epsilon and chitot = chi.  The wake-ellipsoid
// copies (energy_wake.dat) are 0 except tkemean: wakelengthcalc is not
// called (postp.f:36-38), the wake radii stay 0 and no point is inside.
// dumeandz: (2/zh) D umean per subdomain; dumeandy: the real Fourier series of
// umean in y differentiated, without its Nyquist term (the inverse real
// transform drops the imaginary Nyquist coefficient), 0 for ny = 1.
//
// The device reduces every needed product over x into per-(j,k) row sums;
// the host adds the rows in a fixed order, so the result is deterministic.

template <typename T>
__global__ void __launch_bounds__(256) k_row_dot(Geo g, const T* __restrict__ a, const T* __restrict__ b,
                                                 double* __restrict__ out) {
  const int j = blockIdx.x, k = blockIdx.y;
  const size_t base = (size_t)k * g.plane + (size_t)j * g.nxpp;
  double s = 0;
  for (int i = threadIdx.x; i < g.nx; i += blockDim.x) s += (double)a[base + i] * (b ? (double)b[base + i] : 1.0);
  __shared__ double sh[256];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[(size_t)k * g.ny + j] = sh[0];
}

// u' = u - umean with umean = (row sum)/nx for k >= 2 (1-based), 0 at k = 1
template <typename T>
__global__ void k_sub_rowmean(Geo g, T* __restrict__ a, const double* __restrict__ rowsum) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.plane * (size_t)g.nz) return;
  const int i = (int)(t % g.nxpp);
  const size_t r = t / g.nxpp;
  const int j = (int)(r % g.ny), k = (int)(r / g.ny);
  if (i >= g.nx || k == 0) return;
  a[t] = (T)((double)a[t] - rowsum[(size_t)k * g.ny + j] / g.nx);
}

constexpr int kPostpRows = 20;  // row-sum arrays per call

template <typename T>
static int postp_impl(iw_handle* h, FieldSet<T>& fs, double* e18, double* w18) {
  Geo g = geo(h);
  const size_t ny = h->ny, nz = h->nz, rows = ny * nz;
  if (!h->dpostp) {
    const cudaError_t e = cudaMalloc(&h->dpostp, kPostpRows * rows * sizeof(double));
    if (e != cudaSuccess) return set_err(IW_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  double* R = h->dpostp;
  T *pu = fs.X11[0], *pv = fs.X11[1], *pw = fs.X11[2], *pt = fs.X11[3], *su = fs.X11[4];
  T *dst = fs.Y12[0], *tmp = fs.Y12[1];
  const dim3 rg((unsigned)ny, (unsigned)nz);
  T* phys[4] = {pu, pv, pw, pt};
  for (int q = 0; q < 4; ++q) phys_of<T>(h, fs, fs.F[q], phys[q], tmp, 0);
  k_row_dot<T><<<rg, 256, 0, h->st>>>(g, pu, nullptr, R);  // 0: row sums of u
  k_sub_rowmean<T><<<(unsigned)((h->plane * nz + 255) / 256), 256, 0, h->st>>>(g, pu, R);
  // spectral u', v, w, temp: the forward transform of the physical fields, as
  // energycalc_postp takes them (postp.f:466-469) before differentiating
  T* spec[4] = {su, fs.X11[5], fs.X11[6], fs.X11[7]};
  for (int q = 0; q < 4; ++q) {
    CK(cudaMemcpyAsync(spec[q], phys[q], h->ntot * sizeof(T), cudaMemcpyDeviceToDevice, h->st));
    int r = horfft_dev<T>(h, fs, spec[q], -1, (int)nz);
    if (r) return r;
    // the sums use the fields transformed back (postp.f:485-488): the round
    // trip is not the identity for the x-Nyquist column, which it rescales
    phys_of<T>(h, fs, spec[q], phys[q], tmp, 0);
  }
  const T* pairs[7][2] = {{pu, pu}, {pv, pv}, {pw, pw}, {pt, pt}, {pu, pv}, {pu, pw}, {pw, pt}};
  for (int n = 0; n < 7; ++n) k_row_dot<T><<<rg, 256, 0, h->st>>>(g, pairs[n][0], pairs[n][1], R + (1 + n) * rows);
  const T* srcs[4] = {spec[0], spec[1], spec[2], spec[3]};
  for (int s = 0; s < 4; ++s)
    for (int op = 1; op <= 3; ++op) {
      phys_of<T>(h, fs, srcs[s], dst, tmp, op);
      k_row_dot<T><<<rg, 256, 0, h->st>>>(g, dst, dst, R + (8 + 3 * s + op - 1) * rows);
    }
  CK(cudaGetLastError());
  std::vector<double> hr(kPostpRows * rows);
  CK(cudaMemcpyAsync(hr.data(), R, hr.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  auto row = [&](int n, size_t j, size_t k) { return hr[n * rows + k * ny + j]; };
  // umean and its derivatives (small (ny, nz) planes, on the host)
  std::vector<double> um(rows, 0.0), dz(rows, 0.0), dy(rows, 0.0);
  for (size_t k = 1; k < nz; ++k)
    for (size_t j = 0; j < ny; ++j) um[k * ny + j] = row(0, j, k) / h->nx;
  const int N = h->N;
  for (size_t j = 0; j < ny; ++j)
    for (int ks = 0; ks < h->ns; ++ks)
      for (int k1 = 0; k1 < N; ++k1) {
        double s = 0.0;
        for (int k2 = 0; k2 < N; ++k2) s = s + h->tab.D[(size_t)k1 * N + k2] * um[(size_t)(ks * N + k2) * ny + j];
        dz[(size_t)(ks * N + k1) * ny + j] = s * (2. / h->p.zh[ks]);
      }
  if (ny > 1) {
    const double pi2 = 8. * std::atan(1.0), beta = pi2 / h->p.ylen;
    std::vector<double> cs(ny), sn(ny);
    for (size_t m = 0; m < ny; ++m) {
      cs[m] = std::cos(pi2 * (double)m / (double)ny);
      sn[m] = std::sin(pi2 * (double)m / (double)ny);
    }
    const size_t nyh = ny / 2;
    for (size_t k = 0; k < nz; ++k) {
      const double* a = um.data() + k * ny;
      for (size_t m = 1; m < nyh; ++m) {  // A_m = (1/ny) sum_l a_l e^{-i 2 pi l m / ny}
        double re = 0, im = 0;
        for (size_t l = 0; l < ny; ++l) {
          const size_t p = (l * m) % ny;
          re += a[l] * cs[p];
          im -= a[l] * sn[p];
        }
        re /= ny;
        im /= ny;
        const double kre = -(double)m * beta * im, kim = (double)m * beta * re;  // i ky A_m
        for (size_t j = 0; j < ny; ++j) {
          const size_t p = (j * m) % ny;
          dy[k * ny + j] += 2.0 * (kre * cs[p] - kim * sn[p]);
        }
      }
    }
  }
  double s[kPostpRows] = {0};
  double prody = 0, prodz = 0, tkemean = 0;
  for (size_t k = 1; k < nz; ++k)
    for (size_t j = 0; j < ny; ++j) {
      for (int n = 1; n < kPostpRows; ++n) s[n] += row(n, j, k);
      prody += -dy[k * ny + j] * row(5, j, k);
      prodz += -dz[k * ny + j] * row(6, j, k);
      tkemean += um[k * ny + j] * um[k * ny + j];
    }
  const double ra = 0.0, pr = h->p.xnu;
  double eps = 0, chi = 0;
  for (int n = 8; n < 17; ++n) eps += s[n];
  for (int n = 17; n < 20; ++n) chi += s[n];
  const double tketot = 0.5 * (s[1] + s[2] + s[3]);
  const double tt = h->t - h->tstart;
  const double e[18] = {tt,
                        tt * h->p.brunt,
                        tketot,
                        s[1],
                        s[2],
                        s[3],
                        prody,
                        prodz,
                        prody + prodz,
                        s[7] * ra * pr,
                        eps * pr,
                        0.0,
                        eps * pr + 0.0,
                        chi * h->p.xkappa,
                        0.0,
                        0.0 + chi * h->p.xkappa,
                        tkemean * 0.5 * h->nx,
                        s[4]};
  if (e18) std::memcpy(e18, e, sizeof e);
  if (w18) {
    for (int n = 0; n < 18; ++n) w18[n] = 0.0;
    w18[0] = e[0];
    w18[1] = e[1];
    w18[16] = e[16];
  }
  return IW_OK;
}

// postp's output lines: FORMAT (1x,F10.4,17(2x,E12.6)) for energy.dat and
// energy_wake.dat, (1x,F10.4,8(2x,E12.6)) for wakescale.dat (all 0 but the
// times: wakelengthcalc is not called); headers as the reference's own files
// (main.f:298-311).
static int postp_write(iw_handle* h, const double* e18, const double* w18) {
  static const char* kHead =
      " VARIABLES =\"TIME\",\"Nt\",\"TKE\",\"u1tke\",\"u2tke\",\"u3tke\",\"PRODY\",\"PRODZ\",\"PROD\",\"BFLUX\",\"CHI\","
      "\"CHISGS\",\"CHITOT\",\"EPSILON\",\"EPSSGS\",\"EPSTOT\",\"TKEmean\",\"Tvar\"\n";
  static const char* kHeadW = " VARIABLES =\"TIME\",\"Nt\",\"umax\",\"umaxy\",\"umaxz\",\"L_y\",\"L_z\",\"yc\",\"zc\"\n";
  const std::string dir = h->postp_dir.empty() ? std::string() : h->postp_dir + "/";
  struct Out {
    const char* name;
    const char* head;
    int n;
    const double* v;
  };
  double ws[9] = {e18[0], e18[1], 0, 0, 0, 0, 0, 0, 0};
  const Out outs[3] = {{"energy.dat", kHead, 18, e18}, {"energy_wake.dat", kHead, 18, w18}, {"wakescale.dat", kHeadW, 9, ws}};
  for (const Out& o : outs) {
    const std::string path = dir + o.name;
    FILE* f = fopen(path.c_str(), h->postp_started ? "a" : "w");
    if (!f) return set_err(IW_ERR_IO, "cannot open " + path);
    std::string s = h->postp_started ? std::string() : std::string(o.head);
    s += ' ';
    s += fout::f_wd(o.v[0], 10, 4);
    for (int n = 1; n < o.n; ++n) {
      s += "  ";
      s += fout::e12_6(o.v[n]);
    }
    s += '\n';
    const bool ok = fwrite(s.data(), 1, s.size(), f) == s.size();
    if (fclose(f) != 0 || !ok) return set_err(IW_ERR_IO, "write error on " + path);
  }
  h->postp_started = true;
  return IW_OK;
}

template <typename T>
static int postp_step(iw_handle* h, FieldSet<T>& fs) {
  double e[18], w[18];
  int r = postp_impl<T>(h, fs, e, w);
  if (r) return r;
  return postp_write(h, e, w);
}

extern "C" {

int iw_postp(iw_handle* h, double* e18, double* w18) {
  if (!h) return set_err(IW_ERR_STATE, "null handle");
  cudaSetDevice(h->dev);
  return h->mixed ? postp_impl<float>(h, h->f32, e18, w18) : postp_impl<double>(h, h->f64, e18, w18);
}

int iw_set_postp(iw_handle* h, int npostp, double tstart, const char* dir) {
  if (!h) return set_err(IW_ERR_STATE, "null handle");
  h->npostp = npostp > 0 ? npostp : 0;
  h->tstart = tstart;
  h->postp_dir = dir ? dir : "";
  h->postp_started = false;
  return IW_OK;
}

}  // extern "C"
