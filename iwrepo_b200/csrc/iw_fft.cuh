// Shared-memory FFT building blocks for sm_100a.
//
// Complex FFTs of length M (M = 2^a 3^b 5^c) are done as Stockham autosort
// passes (radix 4, 2, 3, 5) on data held in shared memory; a thread block
// works on a batch of independent transforms at once, one butterfly per
// thread per pass.  Real transforms of length N = 2M use the half-length
// complex transform plus the usual even/odd split.  Twiddles come from tables
// built on the host in long double.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace iw {

template <typename T>
struct cplx_t;
template <>
struct cplx_t<double> {
  typedef double2 type;
};
template <>
struct cplx_t<float> {
  typedef float2 type;
};

template <typename C>
__device__ __forceinline__ C cmk(decltype(C().x) a, decltype(C().x) b) {
  C c;
  c.x = a;
  c.y = b;
  return c;
}
template <typename C>
__device__ __forceinline__ C cadd(C a, C b) {
  return cmk<C>(a.x + b.x, a.y + b.y);
}
template <typename C>
__device__ __forceinline__ C csub(C a, C b) {
  return cmk<C>(a.x - b.x, a.y - b.y);
}
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  return cmk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C>
__device__ __forceinline__ C cconj(C a) {
  return cmk<C>(a.x, -a.y);
}
// multiply by -i (forward) or +i (inverse)
template <typename C>
__device__ __forceinline__ C cmul_mi(C a, bool inv) {
  return inv ? cmk<C>(-a.y, a.x) : cmk<C>(a.y, -a.x);
}

// Plan of one complex length; radices in pass order.
struct FftPlan {
  int M;
  int npass;
  int rad[12];
  int ns[12];       // accumulated size before the pass
  int nbsh[12];     // log2(M/R) if a power of two, else -1
  int nssh[12];     // log2(ns) if a power of two, else -1
};

// One Stockham pass over `nb` batched transforms stored contiguously
// (stride M) in src, written to dst.  W[e] = exp(-2 pi i e / M).
template <typename C>
__device__ __forceinline__ void fft_pass(const C* __restrict__ src, C* __restrict__ dst, int M, int R,
                                         int Ns, int nbatch, const C* __restrict__ W, bool inv, int tid,
                                         int nthr, int nbsh, int nssh) {
  const int nb = M / R;
  const int total = nb * nbatch;
  const int step = M / (Ns * R);
  for (int w = tid; w < total; w += nthr) {
    const int b = nbsh >= 0 ? (w >> nbsh) : (w / nb);
    const int j = w - b * nb;
    const C* s = src + (size_t)b * M;
    C* d = dst + (size_t)b * M;
    C v[5];
    const int jq = nssh >= 0 ? (j >> nssh) : (j / Ns);
    const int jm = j - jq * Ns;
#pragma unroll
    for (int r = 0; r < 5; ++r)
      if (r < R) v[r] = s[j + r * nb];
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < 5; ++r)
        if (r < R) {
          C tw = W[r * jm * step];  // r*jm*step < R*Ns*step = M
          if (inv) tw.y = -tw.y;
          v[r] = cmul(v[r], tw);
        }
    }
    C o[5];
    if (R == 4) {
      C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
      C t2 = cadd(v[1], v[3]), t3 = cmul_mi(csub(v[1], v[3]), inv);
      o[0] = cadd(t0, t2);
      o[2] = csub(t0, t2);
      o[1] = cadd(t1, t3);
      o[3] = csub(t1, t3);
    } else if (R == 2) {
      o[0] = cadd(v[0], v[1]);
      o[1] = csub(v[0], v[1]);
    } else {
      const int q0 = M / R;
#pragma unroll
      for (int q = 0; q < 5; ++q)
        if (q < R) {
          C acc = v[0];
#pragma unroll
          for (int p = 1; p < 5; ++p)
            if (p < R) {
              C tw = W[((p * q) % R) * q0];
              if (inv) tw.y = -tw.y;
              acc = cadd(acc, cmul(v[p], tw));
            }
          o[q] = acc;
        }
    }
    const int base = jq * Ns * R + jm;
#pragma unroll
    for (int r = 0; r < 5; ++r)
      if (r < R) d[base + r * Ns] = o[r];
  }
}

// Full transform; returns the buffer (a or b) that holds the result.
// Caller must __syncthreads() before (inputs ready); this ends synced.
template <typename C>
__device__ C* fft_run(C* a, C* b, const FftPlan& pl, int nbatch, const C* W, bool inv, int tid, int nthr) {
  C* src = a;
  C* dst = b;
  for (int p = 0; p < pl.npass; ++p) {
    fft_pass<C>(src, dst, pl.M, pl.rad[p], pl.ns[p], nbatch, W, inv, tid, nthr, pl.nbsh[p], pl.nssh[p]);
    __syncthreads();
    C* t = src;
    src = dst;
    dst = t;
  }
  return src;
}

}  // namespace iw
