// Field dumps: output.f:118-265 (subroutine plotf).  u, v, w and temp are
// transformed to physical space and written with the run time, the dims and
// the grid:
//   iform = 0: unformatted sequential (the framing of the restart files):
//              t | nx, ny, nz, ntot | x(1..nx) | y | z | then u, v, w, temp as
//              REAL*4 over (nxpp, ny, nz), one record each;
//   iform = 1: formatted, FORMAT 5e14.6 for the reals and 5i10 for the dims,
//              the four fields in one list (output.f:214-223).
// The two padding entries of every x row (i = nx+1, nx+2) hold 0, which is
// what the inverse transform of horfft leaves there.  The reference ends
// plotf by transforming the fields back to spectral space, a projection that
// the next step's maxcalc round trip applies anyway; here the state is not
// touched at all.
//
// The dump is asynchronous: the transforms and the copies into a pinned host
// buffer are queued on the handle's stream, and a host thread waits for them
// and writes the file while later steps run.  iw_wait_fields joins it.

namespace fout {

// Fortran Ew.d output for w = 14, d = 6: [-]0.dddddd E[+-]ee, right-justified.
static void e14_6(std::string& s, double v) {
  char cell[32];
  if (std::isnan(v)) {
    snprintf(cell, sizeof cell, "%14s", "NaN");
  } else if (std::isinf(v)) {
    snprintf(cell, sizeof cell, "%14s", v < 0 ? "-Infinity" : "Infinity");
  } else if (v == 0.0) {
    snprintf(cell, sizeof cell, "%14s", std::signbit(v) ? "-0.000000E+00" : "0.000000E+00");
  } else {
    char m[32];
    snprintf(m, sizeof m, "%.5e", std::fabs(v));  // d.ddddde[+-]x..x, correctly rounded
    const int e = atoi(m + 8) + 1;                // exponent of the 0.dddddd form
    char body[32];
    const char* sign = v < 0 ? "-" : "";
    const int ae = e < 0 ? -e : e;
    if (ae <= 99)
      snprintf(body, sizeof body, "%s0.%c%.5sE%c%02d", sign, m[0], m + 2, e < 0 ? '-' : '+', ae);
    else  // three-digit exponents drop the E
      snprintf(body, sizeof body, "%s0.%c%.5s%c%03d", sign, m[0], m + 2, e < 0 ? '-' : '+', ae);
    snprintf(cell, sizeof cell, "%14s", body);
  }
  s += cell;
}

// one formatted WRITE of a list of reals with FORMAT 5e14.6
struct List {
  std::string s;
  int col = 0;
  void real(double v) {
    if (col == 5) {
      s += '\n';
      col = 0;
    }
    e14_6(s, v);
    ++col;
  }
  void end() {
    s += '\n';
    col = 0;
  }
};

struct Job {
  std::string path;
  int iform = 0, dev = 0, nx = 0, ny = 0, nz = 0, nxpp = 0;
  size_t ntot = 0;
  bool fp32 = false;  // the pinned buffer holds float (mixed handles) or double
  double t = 0;
  std::vector<double> x, y, z;
  const void* host = nullptr;
  cudaEvent_t ev = nullptr;
};

static double value(const Job& j, size_t q, size_t p) {
  const size_t i = p % (size_t)j.nxpp;
  if (i >= (size_t)j.nx) return 0.0;
  return j.fp32 ? (double)((const float*)j.host)[q * j.ntot + p] : ((const double*)j.host)[q * j.ntot + p];
}

static bool write_job(const Job& j, std::string* msg) {
  FILE* f = fopen(j.path.c_str(), j.iform == 0 ? "wb" : "w");
  if (!f) {
    *msg = "cannot open " + j.path + " for writing";
    return false;
  }
  bool ok = true;
  if (j.iform == 0) {
    auto rec = [&](const void* d, size_t n) { return rst::put_record(f, d, n); };
    const int32_t dims[4] = {j.nx, j.ny, j.nz, (int32_t)j.ntot};
    ok = rec(&j.t, 8) && rec(dims, sizeof dims) && rec(j.x.data(), 8 * j.x.size()) && rec(j.y.data(), 8 * j.y.size()) &&
         rec(j.z.data(), 8 * j.z.size());
    std::vector<float> buf(j.ntot);
    for (size_t q = 0; q < 4 && ok; ++q) {
      for (size_t p = 0; p < j.ntot; ++p) buf[p] = (float)value(j, q, p);  // real(u(i,j,k)), output.f:158
      ok = rec(buf.data(), 4 * j.ntot);
    }
  } else {
    List l;
    l.real(j.t);
    l.end();
    char c[16];
    for (int v : {j.nx, j.ny, j.nz, (int)j.ntot}) {
      snprintf(c, sizeof c, "%10d", v);
      l.s += c;
    }
    l.s += '\n';
    for (const auto* a : {&j.x, &j.y, &j.z}) {
      for (double v : *a) l.real(v);
      l.end();
    }
    ok = fwrite(l.s.data(), 1, l.s.size(), f) == l.s.size();
    l.s.clear();
    for (size_t q = 0; q < 4 && ok; ++q)
      for (size_t p = 0; p < j.ntot && ok; ++p) {
        l.real(value(j, q, p));
        if (l.s.size() > (1u << 22)) {
          ok = fwrite(l.s.data(), 1, l.s.size(), f) == l.s.size();
          l.s.clear();
        }
      }
    l.end();
    ok = ok && fwrite(l.s.data(), 1, l.s.size(), f) == l.s.size();
  }
  ok = (fclose(f) == 0) && ok;
  if (!ok) *msg = "write error on " + j.path;
  return ok;
}

}  // namespace fout

static int out_join(iw_handle* h) {
  if (!h->out_thread) return IW_OK;
  h->out_thread->join();
  delete h->out_thread;
  h->out_thread = nullptr;
  return h->out_status;
}

// Animation dumps, solver.f:136-222: when t - Tdump >= dtanim at the start of
// convec, file vortanimout_NNNNN.dat (NNNNN = the dump counter, i5.5) holds
//   ' ZONE F=POINT, I=', nx, ', J=', nz          (list-directed: I12 fields,
//                                                 a blank before ', J=')
// then, for ks, kloc, i: x, z, u, w, temp, temp + rhomean(z) in physical
// space, FORMAT (1x,6(F25.16,3x)).  The reference indexes the fields with the
// y loop variable that the loop of solver.f:82-100 leaves behind, j = ny+1:
// u(i,ny+1,k) is u(i,1,k+1), and for k = nz the row after u, w and temp in
// COMMON /flow/: v(i,1,1), temp(i,1,1) and un(i,1,1) (physical, physical,
// and the spectral level n-1).  The same rows are written here.  After each
// file, one line is appended to animdump.log (solver.f:212-215, list-directed:
// t in 15 significant digits of F form between 3 and 6 blanks, I12 integers,
// a blank before a character item that follows a number).
namespace fout {

// t as ifort's list-directed output writes a REAL*8 of magnitude in [1, 1e15):
// 15 significant digits in F form
static std::string list_real15(double v) {
  char e[40], f[64];
  snprintf(e, sizeof e, "%.14e", v);  // 15 significant digits, correctly rounded
  const int ex = atoi(strchr(e, 'e') + 1);
  const int dec = ex >= 14 ? 0 : 14 - ex;
  snprintf(f, sizeof f, "%.*f", dec, v);
  return f;
}

static std::string animdump_line(double t, int n, int istep) {
  char c[128];
  snprintf(c, sizeof c, "      vortanimout_%12d .datat step=%12d\n", n, istep);
  return " Animation data dumped out at time   " + list_real15(t) + c;
}

struct AnimJob {
  std::string path, log;  // the dump file and animdump.log
  double t = 0;
  int n = 0, istep = 0;
  int dev = 0, nx = 0, nz = 0, nxpp = 0;
  bool fp32 = false;
  std::vector<double> x, z;
  double rg = 0;  // rhograd (forcing.f:115-120)
  const void* host = nullptr;
  cudaEvent_t ev = nullptr;
};

static bool write_anim(const AnimJob& j, std::string* msg) {
  FILE* f = fopen(j.path.c_str(), "w");
  if (!f) {
    *msg = "cannot open " + j.path + " for writing";
    return false;
  }
  const size_t row = j.nxpp, nz = j.nz;
  auto at = [&](size_t r, size_t i) -> double {
    return j.fp32 ? (double)((const float*)j.host)[r * row + i] : ((const double*)j.host)[r * row + i];
  };
  std::string s;
  char c[96];
  snprintf(c, sizeof c, " ZONE F=POINT, I=%12d , J=%12d\n", j.nx, j.nz);
  s += c;
  bool ok = true;
  for (size_t k = 0; k < nz && ok; ++k) {
    const double zz = j.z[k];
    // staging rows: u k=1..nz-1 | w | temp | v(k=0) | temp(k=0) | un(k=0)
    const bool last = k + 1 == nz;
    const size_t ru = last ? 3 * (nz - 1) : k, rw = last ? 3 * (nz - 1) + 1 : (nz - 1) + k,
                 rt = last ? 3 * (nz - 1) + 2 : 2 * (nz - 1) + k;
    for (int i = 0; i < j.nx; ++i) {
      const double tt = at(rt, i);
      const double v[6] = {j.x[i], zz, at(ru, i), at(rw, i), tt, tt + (1. + j.rg * zz)};
      s += ' ';
      for (double x : v) {
        snprintf(c, sizeof c, "%25.16f   ", x);
        s += c;
      }
      s += '\n';
    }
    if (s.size() > (1u << 22)) {
      ok = fwrite(s.data(), 1, s.size(), f) == s.size();
      s.clear();
    }
  }
  ok = ok && fwrite(s.data(), 1, s.size(), f) == s.size();
  ok = (fclose(f) == 0) && ok;
  if (!ok) {
    *msg = "write error on " + j.path;
    return false;
  }
  FILE* lf = fopen(j.log.c_str(), "a");  // open(67,file='animdump.log',access='append')
  if (!lf) {
    *msg = "cannot open " + j.log;
    return false;
  }
  const std::string ln = animdump_line(j.t, j.n, j.istep);
  ok = fwrite(ln.data(), 1, ln.size(), lf) == ln.size();
  ok = (fclose(lf) == 0) && ok;
  if (!ok) *msg = "write error on " + j.log;
  return ok;
}

}  // namespace fout

template <typename T>
static int anim_dump(iw_handle* h, FieldSet<T>& fs) {
  if (out_join(h) != IW_OK) {
    h->out_status = IW_OK;
    return set_err(IW_ERR_IO, "the previous dump failed: " + h->out_msg);
  }
  const size_t row = h->nxpp, plane = (size_t)h->nxpp * h->ny, nz = h->nz, es = sizeof(T);
  const size_t need = (3 * (nz - 1) + 3) * row * es;
  if (h->anim_bytes < need) {
    if (h->anim_host) cudaFreeHost(h->anim_host);
    h->anim_host = nullptr;
    h->anim_bytes = 0;
    CK(cudaMallocHost(&h->anim_host, need));
    h->anim_bytes = need;
  }
  if (!h->out_ev) CK(cudaEventCreateWithFlags(&h->out_ev, cudaEventDisableTiming));
  T* dst = fs.Y12[0];
  char* hb = (char*)h->anim_host;
  // Sources: F1, stage A's copy of the state as convec sees it (after the
  // maxcalc round trip, with the mean of w removed, solver.f:64-67); Y12 is
  // free until the y-inverse that follows.
  // rows j = 1 of planes k = 2..nz (0-based: plane k+1, row 0) of u, w, temp
  const int qs[3] = {0, 2, 3};
  for (int n = 0; n < 3; ++n) {
    phys_of<T>(h, fs, fs.F1[qs[n]], dst, fs.Y12[1], 0);
    if (nz > 1)
      CK(cudaMemcpy2DAsync(hb + (size_t)n * (nz - 1) * row * es, row * es, dst + plane, plane * es, row * es, nz - 1,
                           cudaMemcpyDeviceToHost, h->st));
    if (qs[n] == 3)  // temp(i,1,1): the row after w in COMMON /flow/
      CK(cudaMemcpyAsync(hb + (3 * (nz - 1) + 1) * row * es, dst, row * es, cudaMemcpyDeviceToHost, h->st));
  }
  phys_of<T>(h, fs, fs.F1[1], dst, fs.Y12[1], 0);  // v(i,1,1): the row after u
  CK(cudaMemcpyAsync(hb + 3 * (nz - 1) * row * es, dst, row * es, cudaMemcpyDeviceToHost, h->st));
  // un(i,1,1): the row after temp, the spectral level n-1 of u
  CK(cudaMemcpyAsync(hb + (3 * (nz - 1) + 2) * row * es, fs.Fn[0], row * es, cudaMemcpyDeviceToHost, h->st));
  CK(cudaEventRecord(h->out_ev, h->st));
  fout::AnimJob j;
  char name[32];
  snprintf(name, sizeof name, "vortanimout_%05d.dat", h->ianimc);  // fmt (i5.5,a4), solver.f:159-167
  j.path = h->anim_dir.empty() ? std::string(name) : h->anim_dir + "/" + name;
  j.log = h->anim_dir.empty() ? std::string("animdump.log") : h->anim_dir + "/animdump.log";
  j.t = h->t;
  j.n = h->ianimc;
  j.istep = h->istep;
  j.dev = h->dev;
  j.nx = h->nx;
  j.nz = h->nz;
  j.nxpp = h->nxpp;
  j.fp32 = sizeof(T) == 4;
  j.rg = -h->p.rho0 * (h->p.brunt * h->p.brunt) / h->p.grav;
  {
    const double pi2 = 8. * std::atan(1.0), xl = pi2 / (pi2 / h->p.xlen);
    for (int i = 0; i < h->nx; ++i) j.x.push_back(i * xl / h->nx);
    for (int ks = 0; ks < h->ns; ++ks)
      for (int kl = 0; kl < h->N; ++kl) j.z.push_back(h->p.z0[ks] + 0.5 * h->p.zh[ks] * (h->tab.zpts[kl] + 1.0));
  }
  j.host = h->anim_host;
  j.ev = h->out_ev;
  h->out_status = IW_OK;
  h->out_msg.clear();
  h->out_thread = new std::thread([h, j]() {
    cudaSetDevice(j.dev);
    if (cudaEventSynchronize(j.ev) != cudaSuccess) {
      h->out_msg = "the copies of the animation dump failed";
      h->out_status = IW_ERR_CUDA;
      return;
    }
    std::string msg;
    if (!fout::write_anim(j, &msg)) {
      h->out_msg = msg;
      h->out_status = IW_ERR_IO;
    }
  });
  return IW_OK;
}

// Legendre spectra, filtering.f:1110-1221 (speclegencalc) every ncalclegspec
// steps after t += dt, before the interface averaging (main.f:905-910), for
// u, v, w and T: in the x row of physical space at y index nyh (1-based),
// per subdomain, the mean over x of |a_k|, a_k = (k + 1/2) sum_j wg_j f_j
// P_k(z_j) (k < N-1) and (N-1)/2 sum_j ... for the top mode.  File
// speclegen<c><t>.dat, t in F5.3 (F6.3, F7.3, F8.3 from nint(t) = 10, 100,
// 1000), lines (1x,I2,2x,10(e12.6,2x)) with one line per kloc (more than 10
// subdomains continue on the next line, by format reversion).
template <typename T>
__global__ void k_speclegen(Geo g, const T* __restrict__ f, int jrow, const double* __restrict__ wg,
                            const double* __restrict__ alpol, double* __restrict__ out) {
  const int ks = blockIdx.y, N = g.N;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.nx) return;
  double faux[64];
  for (int kl = 0; kl < N; ++kl) faux[kl] = (double)f[(size_t)(ks * N + kl) * g.plane + (size_t)jrow * g.nxpp + i];
  const int nzm = N - 1;
  for (int k = 0; k <= nzm; ++k) {
    double sum = 0.;
    for (int k1 = 0; k1 < N; ++k1) sum = sum + wg[k1] * faux[k1] * alpol[(size_t)k * N + k1];
    const double a = k == nzm ? 0.5 * nzm * sum : (k + 0.5) * sum;
    out[((size_t)ks * g.nx + i) * N + k] = fabs(a);
  }
}

namespace fout {

// Fortran Fw.d (asterisks when the value does not fit)
static std::string f_wd(double v, int w, int d) {
  char b[64];
  snprintf(b, sizeof b, "%.*f", d, v);
  const std::string s(b);
  if ((int)s.size() > w) return std::string(w, '*');
  return std::string(w - s.size(), ' ') + s;
}

// Fortran Ew.6 for w = 12: 0.dddddd E+ee fills all 12 columns
static std::string e12_6(double v) {
  std::string s;
  e14_6(s, v);
  const size_t lead = s.find_first_not_of(' ');
  std::string body = s.substr(lead);
  if (body.size() > 12 && body.compare(0, 3, "-0.") == 0) body = "-" + body.substr(2);  // optional zero dropped
  if (body.size() > 12) return std::string(12, '*');
  return std::string(12 - body.size(), ' ') + body;
}

static std::string speclegen_name(char c, double t) {
  const long n = std::lround(t);
  const int w = n >= 1000 ? 8 : n >= 100 ? 7 : n >= 10 ? 6 : 5;
  return std::string("speclegen") + c + f_wd(t, w, 3) + ".dat";
}

struct LegJob {
  std::string dir;
  int dev = 0, nx = 0, ns = 0, N = 0;
  double t = 0;
  const double* host = nullptr;  // [4][ns][nx][N] |a_k|
  cudaEvent_t ev = nullptr;
};

static bool write_leg(const LegJob& j, std::string* msg) {
  const char names[4] = {'u', 'v', 'w', 'T'};
  const size_t per = (size_t)j.ns * j.nx * j.N;
  for (int q = 0; q < 4; ++q) {
    std::vector<double> spec((size_t)j.ns * j.N, 0.0);  // specout(ks, kloc)
    for (int ks = 0; ks < j.ns; ++ks) {
      for (int i = 0; i < j.nx; ++i)
        for (int k = 0; k < j.N; ++k) spec[(size_t)ks * j.N + k] += j.host[q * per + ((size_t)ks * j.nx + i) * j.N + k];
      for (int k = 0; k < j.N; ++k) spec[(size_t)ks * j.N + k] = spec[(size_t)ks * j.N + k] / j.nx;
    }
    const std::string name = speclegen_name(names[q], j.t);
    const std::string path = j.dir.empty() ? name : j.dir + "/" + name;
    FILE* f = fopen(path.c_str(), "w");
    if (!f) {
      *msg = "cannot open " + path + " for writing";
      return false;
    }
    std::string s;
    char c[16];
    for (int k = 0; k < j.N; ++k) {
      snprintf(c, sizeof c, " %2d  ", k + 1);
      s += c;
      for (int ks = 0; ks < j.ns; ++ks) {
        if (ks > 0) s += (ks % 10 == 0) ? "\n" : "  ";
        s += e12_6(spec[(size_t)ks * j.N + k]);
      }
      s += '\n';
    }
    const bool ok = fwrite(s.data(), 1, s.size(), f) == s.size();
    if (fclose(f) != 0 || !ok) {
      *msg = "write error on " + path;
      return false;
    }
  }
  return true;
}

}  // namespace fout

template <typename T>
static int legspec_dump(iw_handle* h, FieldSet<T>& fs) {
  if (out_join(h) != IW_OK) {
    h->out_status = IW_OK;
    return set_err(IW_ERR_IO, "the previous dump failed: " + h->out_msg);
  }
  const size_t per = (size_t)h->ns * h->nx * h->N;
  if (!h->dlegspec) {
    const cudaError_t e = cudaMalloc(&h->dlegspec, 4 * per * sizeof(double));
    if (e != cudaSuccess) return set_err(IW_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  if (h->leg_bytes < 4 * per * sizeof(double)) {
    if (h->leg_host) cudaFreeHost(h->leg_host);
    h->leg_host = nullptr;
    h->leg_bytes = 0;
    CK(cudaMallocHost(&h->leg_host, 4 * per * sizeof(double)));
    h->leg_bytes = 4 * per * sizeof(double);
  }
  if (!h->out_ev) CK(cudaEventCreateWithFlags(&h->out_ev, cudaEventDisableTiming));
  const int jrow = h->nyh - 1;  // j = nyh (filtering.f:1156); ny >= 2 here
  for (int q = 0; q < 4; ++q) {
    phys_of<T>(h, fs, fs.F[q], fs.Y12[0], fs.Y12[1], 0);
    k_speclegen<T><<<dim3((unsigned)((h->nx + 127) / 128), (unsigned)h->ns), 128, 0, h->st>>>(
        geo(h), fs.Y12[0], jrow, h->dwg, h->dal, h->dlegspec + q * per);
  }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h->leg_host, h->dlegspec, 4 * per * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaEventRecord(h->out_ev, h->st));
  fout::LegJob j;
  j.dir = h->leg_dir;
  j.dev = h->dev;
  j.nx = h->nx;
  j.ns = h->ns;
  j.N = h->N;
  j.t = h->t;
  j.host = (const double*)h->leg_host;
  j.ev = h->out_ev;
  h->out_status = IW_OK;
  h->out_msg.clear();
  h->out_thread = new std::thread([h, j]() {
    cudaSetDevice(j.dev);
    if (cudaEventSynchronize(j.ev) != cudaSuccess) {
      h->out_msg = "the copies of the Legendre spectra failed";
      h->out_status = IW_ERR_CUDA;
      return;
    }
    std::string msg;
    if (!fout::write_leg(j, &msg)) {
      h->out_msg = msg;
      h->out_status = IW_ERR_IO;
    }
  });
  return IW_OK;
}

extern "C" {

int iw_set_speclegen(iw_handle* h, int ncalclegspec, const char* dir) {
  if (!h) return set_err(IW_ERR_STATE, "null handle");
  if (ncalclegspec > 0 && h->ny < 2)
    return set_err(IW_ERR_CONFIG, "Legendre spectra need ny >= 2: the reference reads y index nyh = 0, outside the "
                                  "field, when ny = 1");
  h->nlegspec = ncalclegspec > 0 ? ncalclegspec : 0;
  h->leg_dir = dir ? dir : "";
  return IW_OK;
}

int iw_set_animation(iw_handle* h, double dtanim, const char* dir) {
  if (!h) return set_err(IW_ERR_STATE, "null handle");
  h->dtanim = dtanim > 0 ? dtanim : 0;
  h->anim_dir = dir ? dir : "";
  h->tdump = 0;
  h->ianimc = 0;
  return IW_OK;
}

int iw_write_fields(iw_handle* h, const char* path, int iform) {
  if (!h || !path) return set_err(IW_ERR_STATE, "iw_write_fields: bad argument");
  if (iform != 0 && iform != 1) return set_err(IW_ERR_CONFIG, "iw_write_fields: iform must be 0 or 1");
  if (!rst::little_endian()) return set_err(IW_ERR_CONFIG, "unformatted files are little-endian; this host is not");
  if ((size_t)4 * h->ntot > rst::kMaxRecord)
    return set_err(IW_ERR_CONFIG, "a REAL*4 field record would exceed 2147483639 bytes");
  cudaSetDevice(h->dev);
  if (out_join(h) != IW_OK) {
    h->out_status = IW_OK;
    return set_err(IW_ERR_IO, "the previous field dump failed: " + h->out_msg);
  }
  const size_t esz = h->mixed ? sizeof(float) : sizeof(double);
  const size_t need = 4 * h->ntot * esz;
  if (h->out_bytes < need) {
    if (h->out_host) cudaFreeHost(h->out_host);
    h->out_host = nullptr;
    h->out_bytes = 0;
    CK(cudaMallocHost(&h->out_host, need));
    h->out_bytes = need;
  }
  if (!h->out_ev) CK(cudaEventCreateWithFlags(&h->out_ev, cudaEventDisableTiming));
  for (int q = 0; q < 4; ++q) {
    void* dst = (char*)h->out_host + (size_t)q * h->ntot * esz;
    if (h->mixed) {
      phys_of<float>(h, h->f32, h->f32.F[q], h->f32.Y12[0], h->f32.Y12[1], 0);
      CK(cudaMemcpyAsync(dst, h->f32.Y12[0], h->ntot * esz, cudaMemcpyDeviceToHost, h->st));
    } else {
      phys_of<double>(h, h->f64, h->f64.F[q], h->f64.Y12[0], h->f64.Y12[1], 0);
      CK(cudaMemcpyAsync(dst, h->f64.Y12[0], h->ntot * esz, cudaMemcpyDeviceToHost, h->st));
    }
  }
  CK(cudaEventRecord(h->out_ev, h->st));
  fout::Job j;
  j.path = path;
  j.iform = iform;
  j.dev = h->dev;
  j.nx = h->nx;
  j.ny = h->ny;
  j.nz = h->nz;
  j.nxpp = h->nxpp;
  j.ntot = h->ntot;
  j.fp32 = h->mixed;
  j.t = h->t;
  j.host = h->out_host;
  j.ev = h->out_ev;
  {  // setup.f:136-166 grids
    const double pi2 = 8. * std::atan(1.0), xl = pi2 / (pi2 / h->p.xlen), yl = pi2 / (pi2 / h->p.ylen);
    for (int i = 0; i < h->nx; ++i) j.x.push_back(i * xl / h->nx);
    for (int jj = 0; jj < h->ny; ++jj) j.y.push_back(jj * yl / h->ny);
    for (int ks = 0; ks < h->ns; ++ks)
      for (int kl = 0; kl < h->N; ++kl) j.z.push_back(h->p.z0[ks] + 0.5 * h->p.zh[ks] * (h->tab.zpts[kl] + 1.0));
  }
  h->out_status = IW_OK;
  h->out_msg.clear();
  h->out_thread = new std::thread([h, j]() {
    cudaSetDevice(j.dev);
    if (cudaEventSynchronize(j.ev) != cudaSuccess) {
      h->out_msg = "the copies of the dump failed";
      h->out_status = IW_ERR_CUDA;
      return;
    }
    std::string msg;
    if (!fout::write_job(j, &msg)) {
      h->out_msg = msg;
      h->out_status = IW_ERR_IO;
    }
  });
  return IW_OK;
}

int iw_wait_fields(iw_handle* h) {
  if (!h) return set_err(IW_ERR_STATE, "null handle");
  const int r = out_join(h);
  if (r != IW_OK) {
    h->out_status = IW_OK;
    return set_err(r, "field dump: " + h->out_msg);
  }
  return IW_OK;
}

}  // extern "C"
