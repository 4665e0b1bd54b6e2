// Restart files: output.f:2-117 writes them, restart.f:2-126 reads them, and
// main.f:555-632 sets up the steps that follow a read.
//
// Format: ifort unformatted sequential.  Each record is framed by its byte
// count as a 4-byte little-endian integer, before and after.  REAL items are
// 8 bytes (the reference is built with -autodouble), INTEGER items 4 bytes.
// ifort splits records longer than 2147483639 bytes into subrecords; such
// records are refused here.
//
// The 49 records of output.f, in its order and with its sizes (the dims of
// dim.h, nz2 = nsubd*(nzloc-1)+1 and nsdtype = 1).  What each holds when this
// library writes it:
//   1 t | 2 pr = xnu (main.f:428), ra = 0 (its start-up value, main.f:577)
//   3 nx, ny, nz, nzm, nxppy, ntot, nsubd, nzloc, nsdtype
//   4 alpha, beta | 5 (xw(i), xsq(i)), i = 1..nx | 6 (yw(j), ysq(j))
//   7 x | 8 y | 9 z | 10 zf(1..nz2) | 11 (z0, zh, isubdtype = 1)
//   12 subdlen(1) = zlen*(1/nsubd) | 13 alpol | 14 dalpol | 15 zpts | 16 wg
//   17 d | 18 d2 | 19 d3 | 20 (atpz, btpz, ctpz) | 21 (tubc, tbbc)
//   22 uw, vw, ww | 23 umax | 24 solks | 25-29 the soliton fields
//   30-33 u, v, w, temp at n | 34-37 at n-1 | 38-41 at n-2
//   42-45 the nonlinear terms at n-1 | 46-49 at n-2
// Records 4-22 are setup tables, which the reference computes again right
// after the read (main.f:591 calls setup).  Record 5 runs past xw's bound
// (nxhp) to nx in the reference, which then writes whatever follows xw in
// COMMON /wave/; here those entries are 0.  dalpol, d3 and atpz/btpz/ctpz
// (not used by this library) are written as 0, and so are tubc/tbbc and
// uw/vw/ww, which the step never reads (calcuvwt.f:296-299,655-658 use 0),
// solks and the soliton fields (wavesetup is not called, main.f:871).
//
// After record 49 this library appends one record of its own: the step
// counter, the restart and adaptive-step state and the multistep
// coefficients.  restart.f stops after record 49, so the reference still
// reads the file; IW_RESTART_EXACT uses the extra record to continue a run
// bit for bit.

namespace rst {

constexpr int32_t kMagic = 0x32425749;  // "IWB2"
constexpr int32_t kVersion = 1;
constexpr size_t kMaxRecord = 2147483639;

struct Rec {
  size_t n8, n4;  // REAL*8 and INTEGER*4 items
  size_t bytes() const { return 8 * n8 + 4 * n4; }
};

// output.f:26-108
static std::vector<Rec> layout(size_t nx, size_t ny, size_t nz, size_t nzloc, size_t nsubd) {
  const size_t nxpp = nx + 2, N = nzloc, nz2 = nsubd * (nzloc - 1) + 1, nt = nxpp * ny * nz;
  std::vector<Rec> r = {{1, 0},           {2, 0},           {0, 9},           {2, 0},           {2 * nx, 0},
                        {2 * ny, 0},      {nx, 0},          {ny, 0},          {nz, 0},          {nz2, 0},
                        {2 * nsubd, nsubd}, {1, 0},         {N * N, 0},       {N * N, 0},       {N, 0},
                        {N, 0},           {N * N, 0},       {N * N, 0},       {N * N, 0},       {3 * nz, 0},
                        {2 * nxpp * ny, 0}, {12 * nxpp * ny, 0}, {1, 0},      {1, 0},           {2 * nxpp * nz, 0},
                        {2 * nxpp * nz, 0}, {2 * nxpp * nz, 0}, {nxpp * nz, 0}, {2 * nxpp * nz, 0}};
  for (int i = 0; i < 20; ++i) r.push_back({nt, 0});
  return r;
}
constexpr size_t kExtraBytes = 6 * 4 + 9 * 8;

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

static bool put_marker(FILE* f, size_t bytes) {
  const uint32_t m = (uint32_t)bytes;
  unsigned char b[4] = {(unsigned char)(m & 0xff), (unsigned char)((m >> 8) & 0xff), (unsigned char)((m >> 16) & 0xff),
                        (unsigned char)(m >> 24)};
  return fwrite(b, 1, 4, f) == 4;
}
static bool get_marker(FILE* f, size_t* bytes) {
  unsigned char b[4];
  if (fread(b, 1, 4, f) != 4) return false;
  const uint32_t m = (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
  if (m & 0x80000000u) return false;  // a subrecord: not written by this format's writers
  *bytes = m;
  return true;
}
// one record from a byte image (items already in file order)
static bool put_record(FILE* f, const void* data, size_t bytes) {
  return put_marker(f, bytes) && (bytes == 0 || fwrite(data, 1, bytes, f) == bytes) && put_marker(f, bytes);
}

// Items of a mixed record in file order, little-endian (the host's order on
// x86-64 and AArch64, checked at run time by the callers).
struct Bytes {
  std::vector<unsigned char> b;
  void f8(double v) {
    const size_t o = b.size();
    b.resize(o + 8);
    std::memcpy(b.data() + o, &v, 8);
  }
  void i4(int32_t v) {
    const size_t o = b.size();
    b.resize(o + 4);
    std::memcpy(b.data() + o, &v, 4);
  }
};

static bool little_endian() {
  const uint32_t one = 1;
  unsigned char c;
  std::memcpy(&c, &one, 1);
  return c == 1;
}

}  // namespace rst

// setup.f:132-166 grids and wavenumbers, as the records hold them
static void rst_tables(const iw_handle* h, rst::Bytes* rec /* records 4..12, index 0 = record 4 */) {
  const int nx = h->nx, ny = h->ny, N = h->N, ns = h->ns, nxhp = h->nxhp, nyh = h->nyh;
  const double pi2 = 8. * std::atan(1.0), alpha = pi2 / h->p.xlen, beta = pi2 / h->p.ylen;
  rec[0].f8(alpha);
  rec[0].f8(beta);
  for (int i = 0; i < nx; ++i) {
    const double xw = i < nxhp ? i * alpha : 0.0;
    rec[1].f8(xw);
    rec[1].f8(xw * xw);
  }
  std::vector<double> yw(ny, 0.0);
  for (int j = 1; j <= nyh; ++j) {
    yw[j - 1] = (j - 1) * beta;
    yw[ny - j] = -j * beta;
  }
  for (int j = 0; j < ny; ++j) {
    rec[2].f8(yw[j]);
    rec[2].f8(yw[j] * yw[j]);
  }
  const double xl = pi2 / alpha, yl = pi2 / beta;
  for (int i = 0; i < nx; ++i) rec[3].f8(i * xl / nx);
  for (int j = 0; j < ny; ++j) rec[4].f8(j * yl / ny);
  std::vector<double> zf((size_t)ns * (N - 1) + 2, 0.0);
  for (int ks = 0; ks < ns; ++ks)
    for (int kl = 0; kl < N; ++kl) {
      const double z = h->p.z0[ks] + 0.5 * h->p.zh[ks] * (h->tab.zpts[kl] + 1.0);
      rec[5].f8(z);
      zf[(size_t)ks * (N - 1) + kl + 1] = z;
    }
  for (size_t k = 1; k <= (size_t)ns * (N - 1) + 1; ++k) rec[6].f8(zf[k]);
  for (int ks = 0; ks < ns; ++ks) {
    rec[7].f8(h->p.z0[ks]);
    rec[7].f8(h->p.zh[ks]);
    rec[7].i4(1);
  }
  rec[8].f8(h->p.zlen * (1. / ns));  // setup.f:281,289
}

extern "C" {

int iw_write_restart(iw_handle* h, const char* path) {
  if (!h || !path) return set_err(IW_ERR_STATE, "iw_write_restart: bad argument");
  if (!rst::little_endian()) return set_err(IW_ERR_CONFIG, "restart files are little-endian; this host is not");
  cudaSetDevice(h->dev);
  const auto lay = rst::layout(h->nx, h->ny, h->nz, h->N, h->ns);
  for (size_t r = 0; r < lay.size(); ++r)
    if (lay[r].bytes() > rst::kMaxRecord)
      return set_err(IW_ERR_CONFIG, "restart record " + std::to_string(r + 1) + " would exceed 2147483639 bytes");
  rst::File out;
  out.f = fopen(path, "wb");
  if (!out.f) return set_err(IW_ERR_IO, std::string("cannot open ") + path + " for writing");
  const int N = h->N;
  std::vector<rst::Bytes> rec(lay.size());
  rec[0].f8(h->t);
  rec[1].f8(h->p.xnu);
  rec[1].f8(0.0);
  for (int32_t v : {h->nx, h->ny, h->nz, N - 1, h->nxpp * h->ny, (int32_t)h->ntot, h->ns, N, 1}) rec[2].i4(v);
  rst_tables(h, &rec[3]);
  for (int k = 0; k < N; ++k)
    for (int j = 0; j < N; ++j) rec[12].f8(h->tab.alpol[(size_t)j * N + k]);
  for (int i = 0; i < N; ++i) {
    rec[14].f8(h->tab.zpts[i]);
    rec[15].f8(h->tab.wg[i]);
  }
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < N; ++i) {
      rec[16].f8(h->tab.D[(size_t)i * N + j]);
      rec[17].f8(h->tab.D2[(size_t)i * N + j]);
    }
  rec[22].f8(h->p.umax);
  bool ok = true;
  for (size_t r = 0; r < 29 && ok; ++r) {
    if (rec[r].b.empty()) rec[r].b.assign(lay[r].bytes(), 0);  // zero records (see the file header)
    if (rec[r].b.size() != lay[r].bytes()) return set_err(IW_ERR_STATE, "restart record size mismatch");
    ok = rst::put_record(out.f, rec[r].b.data(), rec[r].b.size());
  }
  // records 30-49: levels n, n-1, n-2, NL n-1, NL n-2; fields u, v, w, temp
  std::vector<double> lev(4 * h->ntot);
  for (int l = 0; l < 5 && ok; ++l) {
    int r = copy_level(h, l, lev.data(), false);
    if (r) return r;
    for (int q = 0; q < 4 && ok; ++q) ok = rst::put_record(out.f, lev.data() + (size_t)q * h->ntot, h->ntot * 8);
  }
  rst::Bytes ex;
  for (int32_t v : {rst::kMagic, rst::kVersion, h->istep, h->ivardt, h->idtstep, h->istart}) ex.i4(v);
  for (double v : {h->p.dt, h->cdt, h->c.fac1, h->c.fac2, h->c.fac3, h->c.bdf1, h->c.bdf2, h->c.bdf3, h->c.bdfv}) ex.f8(v);
  ok = ok && rst::put_record(out.f, ex.b.data(), ex.b.size());
  ok = ok && fflush(out.f) == 0;
  if (!ok) return set_err(IW_ERR_IO, std::string("write error on ") + path);
  return IW_OK;
}

int iw_read_restart(iw_handle* h, const char* path, int mode, double cdtin) {
  if (!h || !path) return set_err(IW_ERR_STATE, "iw_read_restart: bad argument");
  if (mode != IW_RESTART_EXACT && mode != IW_RESTART_REFERENCE)
    return set_err(IW_ERR_CONFIG, "iw_read_restart: mode must be IW_RESTART_EXACT or IW_RESTART_REFERENCE");
  if (mode == IW_RESTART_REFERENCE && !(cdtin > 0))
    return set_err(IW_ERR_CONFIG, "iw_read_restart: cdtin must be positive");
  if (!rst::little_endian()) return set_err(IW_ERR_CONFIG, "restart files are little-endian; this host is not");
  cudaSetDevice(h->dev);
  rst::File in;
  in.f = fopen(path, "rb");
  if (!in.f) return set_err(IW_ERR_IO, std::string("cannot open ") + path);
  const auto lay = rst::layout(h->nx, h->ny, h->nz, h->N, h->ns);
  const std::string name(path);
  auto bad = [&](size_t r, const std::string& what) {
    return set_err(IW_ERR_CONFIG, name + ": record " + std::to_string(r + 1) + ": " + what);
  };
  // pass 1: every record's framing and size, the dims, t and the extra
  // record, seeking over the fields, so that a bad file changes nothing
  double t = 0;
  std::vector<unsigned char> small;
  std::vector<off_t> at(lay.size(), 0);  // offset of each record's data
  for (size_t r = 0; r < lay.size(); ++r) {
    size_t len = 0, len2 = 0;
    if (!rst::get_marker(in.f, &len)) return bad(r, "missing or unreadable record");
    if (len != lay[r].bytes())
      return bad(r, std::to_string(len) + " bytes, expected " + std::to_string(lay[r].bytes()) + " for these dims");
    at[r] = ftello(in.f);
    if (r < 29) {
      small.resize(len);
      if (len && fread(small.data(), 1, len, in.f) != len) return bad(r, "short record");
      if (r == 0) std::memcpy(&t, small.data(), 8);
      if (r == 2) {
        int32_t d[9];
        std::memcpy(d, small.data(), sizeof d);
        const int32_t want[8] = {h->nx, h->ny, h->nz, h->N - 1, h->nxpp * h->ny, (int32_t)h->ntot, h->ns, h->N};
        for (int i = 0; i < 8; ++i)
          if (d[i] != want[i]) {
            std::string got;
            for (int k = 0; k < 8; ++k) got += " " + std::to_string(d[k]);
            return bad(r, "dims (nx ny nz nzm nxppy ntot nsubd nzloc) =" + got + " differ from the handle's");
          }
      }
    } else if (fseeko(in.f, (off_t)len, SEEK_CUR) != 0) {
      return bad(r, "short record");
    }
    if (!rst::get_marker(in.f, &len2) || len2 != len) return bad(r, "trailing byte count differs from the leading one");
  }
  // the continuation record of this library (absent in the reference's files)
  int32_t ei[6] = {0, 0, 0, 0, 0, 0};
  double ed[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  bool extra = false;
  {
    size_t len = 0, len2 = 0;
    if (rst::get_marker(in.f, &len) && len == rst::kExtraBytes) {
      unsigned char b[rst::kExtraBytes];
      if (fread(b, 1, len, in.f) == len && rst::get_marker(in.f, &len2) && len2 == len) {
        std::memcpy(ei, b, sizeof ei);
        std::memcpy(ed, b + sizeof ei, sizeof ed);
        extra = ei[0] == rst::kMagic && ei[1] == rst::kVersion;
      }
    }
  }
  if (mode == IW_RESTART_EXACT && !extra)
    return set_err(IW_ERR_CONFIG, name + ": no continuation record (a file written by the reference): use "
                                         "IW_RESTART_REFERENCE");
  // pass 2: the fields, one level (4 records) at a time
  std::vector<double> lev(4 * h->ntot);
  for (int l = 0; l < 5; ++l) {
    for (int q = 0; q < 4; ++q) {
      const size_t r = 29 + 4 * (size_t)l + q;
      if (fseeko(in.f, at[r], SEEK_SET) != 0 || fread(lev.data() + (size_t)q * h->ntot, 1, lay[r].bytes(), in.f) !=
                                                     lay[r].bytes())
        return bad(r, "read error");
    }
    int r = copy_level(h, l, lev.data(), true);
    if (r) return r;
  }
  int r = iw_upload_state(h, nullptr, nullptr, nullptr, nullptr, nullptr, t, 0);
  if (r) return r;
  h->tdump = 0;  // COMMON /Dump/ of a restarted run (restart.f does not read it)
  h->ianimc = 0;
  if (mode == IW_RESTART_EXACT) {
    h->istep = ei[2];
    h->ivardt = ei[3];
    h->idtstep = ei[4];
    h->istart = ei[5];
    h->p.dt = ed[0];
    h->cdt = ed[1];
    h->c = Coefs{ed[2], ed[3], ed[4], ed[5], ed[6], ed[7], ed[8], ed[0]};
  } else {
    // main.f:563-632 with istart = 1: the loop counts steps from 1 again, and
    // the first step's coefficients are those of a step dt after two of cdt*dt
    h->istart = 1;
    h->cdt = cdtin;
    const double d1 = h->p.dt, d2 = cdtin * h->p.dt, d3 = cdtin * h->p.dt;
    h->c = Coefs{abvar1_(&d1, &d2, &d3),  abvar2_(&d1, &d2, &d3),  abvar3_(&d1, &d2, &d3),  bdfvar1_(&d1, &d2, &d3),
                 bdfvar2_(&d1, &d2, &d3), bdfvar3_(&d1, &d2, &d3), bdfvarv_(&d1, &d2, &d3), h->p.dt};
  }
  return IW_OK;
}

}  // extern "C"
