// Shared-memory FFT building blocks for sm_100a.
//
// Complex FFTs of length M (M = 2^a 3^b 5^c) are done as Stockham autosort
// passes (radix 8, 4, 2, 3, 5; the power-of-two radices are
// in-register DFTs) on data held in shared memory; a thread block
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

// Asynchronous global -> shared copy of one complex value (8 or 16 bytes,
// naturally aligned), so that a CTA can put all of its loads in flight before
// waiting once.
template <typename C>
__device__ __forceinline__ void cp_async_c(C* smem, const C* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  if (sizeof(C) == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
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

// v * w with w = c - i s (forward) or c + i s (inverse)
template <typename C>
__device__ __forceinline__ C crot(C v, decltype(C().x) c, decltype(C().x) s, bool inv) {
  const decltype(C().x) t = inv ? s : -s;
  return cmk<C>(v.x * c - v.y * t, v.x * t + v.y * c);
}

// In-register DFT of v[0..R-1] (natural order in and out) for R = 2, 4, 8.
// R = 8 is split 2x4 (n = a + 2b, k = c + 4d); h = cos(pi/4).
template <typename C>
__device__ __forceinline__ void dft4(C& a0, C& a1, C& a2, C& a3, bool inv) {
  C t0 = cadd(a0, a2), t1 = csub(a0, a2);
  C t2 = cadd(a1, a3), t3 = cmul_mi(csub(a1, a3), inv);
  a0 = cadd(t0, t2);
  a2 = csub(t0, t2);
  a1 = cadd(t1, t3);
  a3 = csub(t1, t3);
}

template <typename C, int R>
__device__ __forceinline__ void dft_reg(C* v, bool inv) {
  typedef decltype(C().x) T;
  const T h = (T)0.70710678118654752440;   // cos(pi/4)
  if (R == 2) {
    C t = v[0];
    v[0] = cadd(t, v[1]);
    v[1] = csub(t, v[1]);
  } else if (R == 4) {
    dft4(v[0], v[1], v[2], v[3], inv);
  } else if (R == 8) {
    // a in {0,1}: DFT4 over v[a + 2b]
    dft4(v[0], v[2], v[4], v[6], inv);
    dft4(v[1], v[3], v[5], v[7], inv);
    // twiddle w8^c on the a = 1 half (c = 1..3 sit at v[3], v[5], v[7])
    v[3] = crot(v[3], h, h, inv);
    v[5] = cmul_mi(v[5], inv);
    v[7] = crot(v[7], -h, h, inv);
    C o[8];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      o[c] = cadd(v[2 * c], v[2 * c + 1]);
      o[c + 4] = csub(v[2 * c], v[2 * c + 1]);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = o[i];
  }
}

// One Stockham pass of radix R over `nbatch` transforms stored contiguously
// (stride M) in src, written to dst.  W[e] = exp(-2 pi i e / M).
template <typename C, int R>
__device__ __forceinline__ void fft_pass_r(const C* __restrict__ src, C* __restrict__ dst, int M, int Ns, int nbatch,
                                           const C* __restrict__ W, bool inv, int tid, int nthr, int nbsh, int nssh) {
  const int nb = M / R;
  const int total = nb * nbatch;
  const int step = M / (Ns * R);
  for (int w = tid; w < total; w += nthr) {
    const int b = nbsh >= 0 ? (w >> nbsh) : (w / nb);
    const int j = w - b * nb;
    const C* s = src + (size_t)b * M;
    C* d = dst + (size_t)b * M;
    C v[R];
    const int jq = nssh >= 0 ? (j >> nssh) : (j / Ns);
    const int jm = j - jq * Ns;
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = s[j + r * nb];
    if (Ns > 1) {
      const int e = jm * step;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        C tw = W[r * e];  // r*jm*step < R*Ns*step = M
        if (inv) tw.y = -tw.y;
        v[r] = cmul(v[r], tw);
      }
    }
    if (R == 3 || R == 5) {
      const int q0 = M / R;
      C o[R];
#pragma unroll
      for (int q = 0; q < R; ++q) {
        C acc = v[0];
#pragma unroll
        for (int p = 1; p < R; ++p) {
          C tw = W[((p * q) % R) * q0];
          if (inv) tw.y = -tw.y;
          acc = cadd(acc, cmul(v[p], tw));
        }
        o[q] = acc;
      }
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = o[r];
    } else {
      dft_reg<C, R>(v, inv);
    }
    const int base = jq * Ns * R + jm;
#pragma unroll
    for (int r = 0; r < R; ++r) d[base + r * Ns] = v[r];
  }
}

// Full transform; returns the buffer (a or b) that holds the result.
// Caller must __syncthreads() before (inputs ready); this ends synced.
template <typename C>
__device__ C* fft_run(C* a, C* b, const FftPlan& pl, int nbatch, const C* W, bool inv, int tid, int nthr) {
  C* src = a;
  C* dst = b;
  for (int p = 0; p < pl.npass; ++p) {
    const int R = pl.rad[p], Ns = pl.ns[p], bs = pl.nbsh[p], ss = pl.nssh[p];
    switch (R) {
      case 8: fft_pass_r<C, 8>(src, dst, pl.M, Ns, nbatch, W, inv, tid, nthr, bs, ss); break;
      case 4: fft_pass_r<C, 4>(src, dst, pl.M, Ns, nbatch, W, inv, tid, nthr, bs, ss); break;
      case 2: fft_pass_r<C, 2>(src, dst, pl.M, Ns, nbatch, W, inv, tid, nthr, bs, ss); break;
      case 3: fft_pass_r<C, 3>(src, dst, pl.M, Ns, nbatch, W, inv, tid, nthr, bs, ss); break;
      default: fft_pass_r<C, 5>(src, dst, pl.M, Ns, nbatch, W, inv, tid, nthr, bs, ss); break;
    }
    __syncthreads();
    C* t = src;
    src = dst;
    dst = t;
  }
  return src;
}


// ---------------------------------------------------------------------------
// Warp-synchronous in-place transforms.  One warp owns one transform of length
// M held in shared memory with one pad slot after every 16 values (index
// fpad(i)), which keeps the strided Stockham stores free of bank conflicts.
// Every pass loads all of its butterflies into registers, then stores them:
// no second buffer and no CTA-wide barrier.  DPT >= M/32 values per lane.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ int fpad(int i) { return i + (i >> 4); }
// slots needed for L padded values
__host__ __device__ __forceinline__ int fpadlen(int L) { return L > 0 ? fpad(L - 1) + 1 : 0; }

template <typename C, int R, int NB>
__device__ __forceinline__ void fft_pass_w(C* row, int M, int Ns, const C* __restrict__ W, bool inv, int lane,
                                           int nssh) {
  const int nb = M / R;
  const int step = M / (Ns * R);
  C v[NB][R];
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    const int j = lane + 32 * q;
    if (j < nb) {
      const int jq = nssh >= 0 ? (j >> nssh) : (j / Ns);
      const int jm = j - jq * Ns;
#pragma unroll
      for (int r = 0; r < R; ++r) v[q][r] = row[fpad(j + r * nb)];
      if (Ns > 1) {
        const int e = jm * step;
#pragma unroll
        for (int r = 1; r < R; ++r) {
          C tw = W[r * e];
          if (inv) tw.y = -tw.y;
          v[q][r] = cmul(v[q][r], tw);
        }
      }
      if (R == 3 || R == 5) {
        const int q0 = M / R;
        C o[R];
#pragma unroll
        for (int qq = 0; qq < R; ++qq) {
          C acc = v[q][0];
#pragma unroll
          for (int p = 1; p < R; ++p) {
            C tw = W[((p * qq) % R) * q0];
            if (inv) tw.y = -tw.y;
            acc = cadd(acc, cmul(v[q][p], tw));
          }
          o[qq] = acc;
        }
#pragma unroll
        for (int r = 0; r < R; ++r) v[q][r] = o[r];
      } else {
        dft_reg<C, R>(v[q], inv);
      }
    }
  }
  __syncwarp();
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    const int j = lane + 32 * q;
    if (j < nb) {
      const int jq = nssh >= 0 ? (j >> nssh) : (j / Ns);
      const int jm = j - jq * Ns;
      const int base = jq * Ns * R + jm;
#pragma unroll
      for (int r = 0; r < R; ++r) row[fpad(base + r * Ns)] = v[q][r];
    }
  }
  __syncwarp();
}

// In-place transform of one padded row by one warp (all lanes call it).
// POW2: the length is a power of two, so only radix 8, 4, 2 passes are
// compiled (every compiled radix raises the register count of the kernel).
template <typename C, int DPT, bool POW2>
__device__ __forceinline__ void fft_warp(C* row, const FftPlan& pl, const C* __restrict__ W, bool inv, int lane) {
  for (int p = 0; p < pl.npass; ++p) {
    const int Ns = pl.ns[p], ss = pl.nssh[p];
    switch (pl.rad[p]) {
      case 8: fft_pass_w<C, 8, (DPT + 7) / 8>(row, pl.M, Ns, W, inv, lane, ss); break;
      case 4: fft_pass_w<C, 4, (DPT + 3) / 4>(row, pl.M, Ns, W, inv, lane, ss); break;
      case 2: fft_pass_w<C, 2, (DPT + 1) / 2>(row, pl.M, Ns, W, inv, lane, ss); break;
      default:
        if (!POW2) {
          if (pl.rad[p] == 3)
            fft_pass_w<C, 3, (DPT + 2) / 3>(row, pl.M, Ns, W, inv, lane, ss);
          else
            fft_pass_w<C, 5, (DPT + 4) / 5>(row, pl.M, Ns, W, inv, lane, ss);
        }
        break;
    }
  }
}

// minimum resident CTAs of 256 threads for a warp-transform kernel
template <typename T, int DPT>
struct FftOcc {
  static constexpr int v = sizeof(T) == 4 ? (DPT <= 8 ? 4 : DPT <= 16 ? 2 : 1) : (DPT <= 4 ? 4 : DPT <= 8 ? 2 : 1);
};


// ---------------------------------------------------------------------------
// Compile-time plans for power-of-two lengths M (same passes as make_plan:
// ceil(log2 M / 3) passes of radix <= 8, bits spread evenly).  Strides,
// twiddle steps and lane guards become constants.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int ct_log2(int v) { return v <= 1 ? 0 : 1 + ct_log2(v / 2); }
template <int M>
struct CtPlan {
  static constexpr int a = ct_log2(M);
  static constexpr int np = (a + 2) / 3;
  __host__ __device__ static constexpr int bits(int q) { return a / np + (q < a % np ? 1 : 0); }
};

template <typename C, int M, int R, int NS>
__device__ __forceinline__ void fft_pass_ct(C* row, const C* __restrict__ W, bool inv, int lane) {
  constexpr int nb = M / R;
  constexpr int step = M / (NS * R);
  constexpr int NB = (nb + 31) / 32;
  C v[NB][R];
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    const int j = lane + 32 * q;
    if (nb % 32 == 0 || j < nb) {
      const int jm = j & (NS - 1);
#pragma unroll
      for (int r = 0; r < R; ++r) v[q][r] = row[fpad(j + r * nb)];
      if (NS > 1) {
        const int e = jm * step;
#pragma unroll
        for (int r = 1; r < R; ++r) {
          C tw = W[r * e];
          if (inv) tw.y = -tw.y;
          v[q][r] = cmul(v[q][r], tw);
        }
      }
      dft_reg<C, R>(v[q], inv);
    }
  }
  __syncwarp();
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    const int j = lane + 32 * q;
    if (nb % 32 == 0 || j < nb) {
      const int jq = j / NS, jm = j & (NS - 1);
      const int base = jq * NS * R + jm;
#pragma unroll
      for (int r = 0; r < R; ++r) row[fpad(base + r * NS)] = v[q][r];
    }
  }
  __syncwarp();
}

template <typename C, int M, int P, int NS>
__device__ __forceinline__ void fft_passes_ct(C* row, const C* __restrict__ W, bool inv, int lane) {
  if constexpr (P < CtPlan<M>::np) {
    constexpr int R = 1 << CtPlan<M>::bits(P);
    fft_pass_ct<C, M, R, NS>(row, W, inv, lane);
    fft_passes_ct<C, M, P + 1, NS * R>(row, W, inv, lane);
  }
}

// Passes P .. PEND-1 only (the first or last pass run elsewhere).
template <typename C, int M, int P, int PEND, int NS>
__device__ __forceinline__ void fft_passes_ct_to(C* row, const C* __restrict__ W, bool inv, int lane) {
  if constexpr (P < PEND) {
    constexpr int R = 1 << CtPlan<M>::bits(P);
    fft_pass_ct<C, M, R, NS>(row, W, inv, lane);
    fft_passes_ct_to<C, M, P + 1, PEND, NS * R>(row, W, inv, lane);
  }
}

// In-place transform of one padded row of power-of-two length M by one warp.
template <typename C, int M>
__device__ __forceinline__ void fft_warp_ct(C* row, const C* __restrict__ W, bool inv, int lane) {
  fft_passes_ct<C, M, 0, 1>(row, W, inv, lane);
}

}  // namespace iw
