// Device kernels of the time step (sm_100a).
//
// Data layout in HBM (the reference's COMMON layout): a field is
// [nz][ny][nxpp] values, x fastest; in spectral space pairs (Re,Im) for
// kx = 0..nx/2.  "(kx,y) space" is the same layout after the y transform was
// undone (x still spectral).  Storage type T is double (FP64 path) or float
// (mixed path); the band solves always compute in double.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "iw_fft.cuh"

namespace iw {

constexpr int kMaxN = 64;  // max GLL points per subdomain

// Everything a kernel needs to know about one run (passed by value).
struct Geo {
  int nx, ny, nz, N, ns, nxpp, nxh, nxhp, nyh;
  size_t plane;  // nxpp*ny
  size_t ntot;   // plane*nz
  double scaley; // 1/ny
  double dt;
  const double* D;     // N*N row major, D(k,j)
  const double* Lfil;  // N*N precombined Legendre filter (rows: output point)
  const double* hfac;  // ns: 2/zh(ks)
  const double* xw;    // nxhp
  const double* yw;    // ny
  const double* cfour; // ncol: Fourier filter factor per (ii,j) column (j-major)
  const double* zg;    // nz grid
};

template <typename T>
__device__ __forceinline__ size_t fidx(const Geo& g, int i, int j, int k) {
  return (size_t)i + (size_t)g.nxpp * ((size_t)j + (size_t)g.ny * (size_t)k);
}

}  // namespace iw
