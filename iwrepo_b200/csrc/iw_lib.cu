// B200 time step of the stratified Boussinesq solver (Fourier x,y /
// Legendre multidomain penalty z) and its C ABI (include/iw_b200.h).
//
// One step (main.f:653-1066) on device-resident fields:
//   K_A  k_stageA(_r)  maxcalc/convec round-trip projection, w mean = 0,
//                      z-derivatives of u,v,w,rho                   (z columns)
//   K_B  k_yfft        y-inverse of u,v,w,rho, dz, and i ky (.)      (planes)
//   K_C  k_xrow_nl     x-inverse of 16 rows -> skew-symmetric products,
//                      buoyancy, upwind interface penalty, paddle ->
//                      x-forward with i kx folded in                 (rows)
//   K_D  k_yfft        y-forward with i ky folded in                 (planes)
//   K_E  k_stageE(_r)  S = B + dz(Z), SS extrapolation, BDF u*, history,
//                      Fourier x Legendre filter (k_stageE_f32: the
//                      tiled kernel for FP32 fields)                 (z columns)
//        k_wviscrot    rotational viscous pressure BC                (walls)
//   K_F  k_solve_cta   pressure Poisson (divergence, solve, filter, projection)
//        k_solve_cta   u,v / w / rho Helmholtz solves, filters, mean mode
//                      (block inverses; k_press_g / k_visc with the band LU
//                      when the handle asks for the reference's LU)
//   K_H  interface averaging: planes next to interfaces go to physical space,
//        the averaging change comes back; every plane gets the spectral effect
//        of the round trip.
// Around the step (iw_restart.inl, iw_output.inl, iw_postp.inl): the adaptive
// time step's CFL numbers (k_phys_stats), restart files, field and animation
// dumps, Legendre spectra (k_speclegen) and the TKE budget (k_row_dot,
// k_sub_rowmean), written by a host thread from pinned buffers.
// The penalty systems (penalty.f + band_lu.f) are assembled on the device
// (k_factor) when epsilon changes (steps 1-3 and a dt change), one per distinct
// kx^2+ky^2 and system type, then factored (band LU) or turned into block
// inverses of their distinct subdomain blocks.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/iw_b200.h"
#include "iw_fft.cuh"
#include "iw_kernels.cuh"

using namespace iw;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;
static thread_local int g_status = 0;
static int set_err(int code, const std::string& msg) {
  g_err = msg;
  g_status = code;
  return code;
}
#define CK(x)                                                                            \
  do {                                                                                   \
    cudaError_t e_ = (x);                                                                \
    if (e_ != cudaSuccess) return set_err(IW_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// ---------------------------------------------------------------------------
// small device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }

template <typename T>
__device__ __forceinline__ T ld(const T* p) {
  return __ldg(p);
}

// ===========================================================================
// K_A: round-trip projection + w(1,1,:)=0 + z derivatives.
// Thread per (real x index i, y index j, subdomain ks, field q).
// Inputs F (spectral state n); outputs F1 = P(F) (w mean zeroed) and dz(F1).
// P is the exact effect of horfft(+1) followed by horfft(-1) (maxcalc,
// various.f:726-729,848-851): the kx=0 column becomes Hermitian in ky, the
// x-Nyquist column keeps its real part divided by ny, all else is unchanged.
// ===========================================================================
template <typename T>
__device__ __forceinline__ T proj_val(const Geo& g, const T* __restrict__ f, int i, int j, int k) {
  if (i < 2) {
    int jp = (g.ny - j) % g.ny;
    T a = f[fidx<T>(g, i, j, k)];
    T b = f[fidx<T>(g, i, jp, k)];
    return i == 0 ? (T)0.5 * (a + b) : (T)0.5 * (a - b);
  }
  if (i >= g.nx) {
    return i == g.nx ? f[fidx<T>(g, i, j, k)] * (T)g.scaley : (T)0;
  }
  return f[fidx<T>(g, i, j, k)];
}

// Roundings written out (no contraction left to the compiler): the tiled and
// register-column stage A give the same bits whatever their loop structure.
__device__ __forceinline__ float fma_t(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float mul_t(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_t(double a, double b) { return __dmul_rn(a, b); }

// Asynchronous bulk copies into shared memory, completed on an mbarrier;
// every wait is bounded by the global timer.
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// global -> shared bulk copy (16-byte aligned addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// wait for phase `ph` of an mbarrier, for at most `limit_ns`; false if it gave up
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t ph, uint64_t limit_ns) {
  const uint64_t t0 = global_ns();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(ph)
        : "memory");
    if (ok) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
}

// Tiled z-column kernels: a block owns 32 consecutive real x indices of one
// (y index, subdomain) and keeps the N x 32 tile in shared memory; the N x N
// operators (D, filter) are applied with compact loops over the tile.
constexpr int kTX = 32;   // x points per tile (one warp wide)
constexpr int kTW = 8;    // warps per block

template <typename T>
__global__ void __launch_bounds__(kTX* kTW) k_stageA(Geo g, const T* __restrict__ F0, const T* __restrict__ F1_,
                                                     const T* __restrict__ F2_, const T* __restrict__ F3_,
                                                     T* __restrict__ O0, T* __restrict__ O1, T* __restrict__ O2,
                                                     T* __restrict__ O3, T* __restrict__ Z0, T* __restrict__ Z1,
                                                     T* __restrict__ Z2, T* __restrict__ Z3, int proj,
                                                     int* __restrict__ err) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int N = g.N;
  T* sD = (T*)smraw;             // N*N
  T* tile = sD + N * N;          // N*kTX
  for (int t = threadIdx.x; t < N * N; t += blockDim.x) sD[t] = (T)g.D[t];
  const int q = blockIdx.z;
  const T* F = q == 0 ? F0 : q == 1 ? F1_ : q == 2 ? F2_ : F3_;
  T* O = q == 0 ? O0 : q == 1 ? O1 : q == 2 ? O2 : O3;
  T* Z = q == 0 ? Z0 : q == 1 ? Z1 : q == 2 ? Z2 : Z3;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i = blockIdx.x * kTX + lane;
  const int j = blockIdx.y % g.ny, ks = blockIdx.y / g.ny;
  const bool act = i < g.nxpp;
  for (int k = w; k < N; k += kTW) {
    const int kk = ks * N + k;
    T x = 0;
    if (act) {
      x = proj ? proj_val<T>(g, F, i, j, kk) : F[fidx<T>(g, i, j, kk)];
      if (!isfinite(x)) err[0] = 1;  // the state of the last step holds a NaN or Inf
      if (q == 2 && j == 0 && i < 2) x = (T)0;  // wc(1,1,:) = 0, solver.f:66-69
      O[fidx<T>(g, i, j, kk)] = x;
    }
    tile[k * kTX + lane] = x;
  }
  __syncthreads();
  if (!act) return;
  const T fac = (T)g.hfac[ks];
  for (int k1 = w; k1 < N; k1 += kTW) {
    const T* dr = sD + k1 * N;
    T s = 0;
#pragma unroll 4
    for (int k2 = 0; k2 < N; ++k2) s = fma_t(dr[k2], tile[k2 * kTX + lane], s);
    Z[fidx<T>(g, i, j, ks * N + k1)] = mul_t(s, fac);
  }
}

// ===========================================================================
// y transforms (CFFT99 semantics, horfft.f:21-30,51-57): LOT = nx/2 columns,
// the x-Nyquist column is never transformed; forward is scaled by 1/ny (the
// Nyquist column too).  One CTA per (plane, tile of TX kx columns, job).
// Job modes:
//   0 inverse:  dst = Yinv(src)
//   1 inverse:  dst = Yinv(i ky src)
//   2 forward:  dst = Yfwd(src)/ny
//   3 forward:  dst = Yfwd(src)/ny + i ky Yfwd(src2)/ny
// ===========================================================================
template <typename T>
struct YJob {
  const T* src;
  const T* src2;
  T* dst;
  int mode;
};
template <typename T>
struct YJobs {
  YJob<T> j[16];
};

// slots per padded y column: >= fpadlen(ny) and = 2 (mod 16), so that the
// TX columns of a tile sit in different banks
__host__ __device__ __forceinline__ int ystride(int ny) {
  int s = fpadlen(ny);
  return s + ((2 - s) % 16 + 16) % 16;
}

template <typename T, int TX, int DPT, bool POW2, int MC = 0>
__global__ void __launch_bounds__(256, (FftOcc<T, DPT>::v)) k_yfft(Geo g, YJobs<T> jobs, int nplanes, FftPlan pl,
                                              const typename cplx_t<T>::type* __restrict__ Wy) {
  typedef typename cplx_t<T>::type C;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int ny = MC > 0 ? MC : g.ny;  // a constant with a compile-time plan
  const int RSY = ystride(ny);
  C* A = (C*)smraw;
  C* A2 = A + (size_t)TX * RSY;
  const YJob<T> jb = jobs.j[blockIdx.z];
  const int k = blockIdx.y;
  const int ii0 = blockIdx.x * TX;
  const bool fwd = jb.mode >= 2;
  const bool two = jb.mode == 3;
  (void)nplanes;
  // load: column ii0+b, row j -> A[b*RSY + fpad(j)] (all copies in flight at once).
  // With 256 threads and TX | 256 a thread keeps its column b and steps j by
  // JS = 256/TX, so both addresses advance by fixed strides.
  constexpr int JS = 256 / TX;
  static_assert(JS % 16 == 0, "the padded smem stride of a j step must be a constant");
  const int tb = threadIdx.x % TX, tj = threadIdx.x / TX;
  const int iit = ii0 + tb;
  const bool colok = iit < g.nxhp;
  const size_t gstep = (size_t)JS * g.nxpp;
  // mode 1 with a compile-time length: the i ky factor is applied as the
  // values arrive (plain loads, all in flight), not in a second pass over the
  // shared tile
  constexpr bool kyload = MC > 0 && MC % JS == 0;
  const bool mulky = kyload && jb.mode == 1;
  // With a compile-time plan whose first pass has nb0 = MC / R0 butterflies, a
  // multiple of JS, a thread's loaded values (rows tj + JS it) hold every input
  // of its first-pass butterflies (rows j + nb0 r, j = tj + JS m).  The first
  // Stockham pass (Ns = 1, no twiddles) then runs in registers as the values
  // arrive, and the warps start at the second pass: one shared-memory write and
  // one read less per value.  The x-Nyquist column keeps its raw values.
  constexpr int R0 = MC > 0 ? 1 << CtPlan<(MC > 0 ? MC : 2)>::bits(0) : 1;
  constexpr int NB0 = MC > 0 ? MC / R0 : 1;
  constexpr bool fuse1 = MC > 0 && R0 <= 8 && NB0 % JS == 0 && CtPlan<(MC > 0 ? MC : 2)>::np > 1;
  // Likewise the last pass (Ns = MC / RL, as many butterflies): butterfly j
  // writes rows j + Ns r, all of them rows of the thread with tj = j mod JS
  // when Ns is a multiple of JS, so it runs as the values are stored.
  constexpr int NPS = CtPlan<(MC > 0 ? MC : 2)>::np;
  constexpr int RL = MC > 0 ? 1 << CtPlan<(MC > 0 ? MC : 2)>::bits(NPS - 1) : 1;
  constexpr int NSL = MC > 0 ? MC / RL : 1;
  constexpr bool fuseL = fuse1 && NPS >= 2 && RL <= 8 && NSL % JS == 0;
  if constexpr (fuse1) {
    constexpr int NIT = MC / JS, NBT = NB0 / JS;
    const bool tr = iit < g.nxh;
    const size_t g0 = fidx<T>(g, 2 * iit, tj, k);
#pragma unroll 1
    for (int hh = 0; hh < (two ? 2 : 1); ++hh) {
      const C* s1 = (const C*)((hh ? jb.src2 : jb.src) + g0);
      C* row = (hh ? A2 : A) + tb * RSY;
      C v[NIT];
#pragma unroll
      for (int it = 0; it < NIT; ++it) v[it] = colok ? s1[(size_t)it * (gstep / 2)] : cmk<C>(0, 0);
      if (jb.mode == 1) {
#pragma unroll
        for (int it = 0; it < NIT; ++it) {
          const T ky = (T)g.yw[tj + it * JS];
          v[it] = cmk<C>(-(ky * v[it].y), ky * v[it].x);
        }
      }
      if (tr) {
#pragma unroll
        for (int mb = 0; mb < NBT; ++mb) {
          C w[R0];
#pragma unroll
          for (int r = 0; r < R0; ++r) w[r] = v[mb + r * NBT];  // row tj + JS mb + NB0 r
          dft_reg<C, R0>(w, !fwd);
          const int b0 = (tj + JS * mb) * R0;
#pragma unroll
          for (int r = 0; r < R0; ++r) row[fpad(b0 + r)] = w[r];
        }
      } else {
#pragma unroll
        for (int it = 0; it < NIT; ++it) row[fpad(tj) + it * (JS + JS / 16)] = v[it];
      }
    }
  } else if (mulky) {
    const size_t g0 = fidx<T>(g, 2 * iit, tj, k);
    C* d = A + tb * RSY + fpad(tj);
    const C* s1 = (const C*)(jb.src + g0);
    C v[kyload ? MC / JS : 1];
#pragma unroll
    for (int it = 0; it < (kyload ? MC / JS : 1); ++it)
      v[it] = colok ? s1[(size_t)it * (gstep / 2)] : cmk<C>(0, 0);
#pragma unroll
    for (int it = 0; it < (kyload ? MC / JS : 1); ++it) {
      const T ky = (T)g.yw[tj + it * JS];
      d[it * (JS + JS / 16)] = cmk<C>(-(ky * v[it].y), ky * v[it].x);
    }
  } else {
    const size_t g0 = fidx<T>(g, 2 * iit, tj, k);
    C* d = A + tb * RSY + fpad(tj);
    const C* s1 = (const C*)(jb.src + g0);
    const C* s2 = two ? (const C*)(jb.src2 + g0) : s1;
    for (int j = tj; j < ny; j += JS) {
      if (colok) {
        cp_async_c<C>(d, s1);
        if (two) cp_async_c<C>(d + TX * RSY, s2);
      } else {
        *d = cmk<C>(0, 0);
        if (two) d[TX * RSY] = cmk<C>(0, 0);
      }
      d += JS + JS / 16;
      s1 = (const C*)((const T*)s1 + gstep);
      s2 = (const C*)((const T*)s2 + gstep);
    }
  }
  cp_async_wait_all();
  __syncthreads();
  if (jb.mode == 1 && !mulky) {
    for (int t = threadIdx.x; t < TX * ny; t += blockDim.x) {
      const int b = t % TX, j = t / TX;
      const T ky = (T)g.yw[j];
      C* d = A + b * RSY + fpad(j);
      const C v = *d;
      *d = cmk<C>(-(ky * v.y), ky * v.x);
    }
    __syncthreads();
  }
  // the x-Nyquist column (ii = nxh) is not transformed
  const int nb = ny > 1 ? max(0, min(TX, g.nxh - ii0)) : 0;
  const int nrow = two ? 2 * nb : nb;
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int r = threadIdx.x >> 5; r < nrow; r += nw) {
    C* row = r < nb ? A + r * RSY : A2 + (r - nb) * RSY;
    if constexpr (fuseL)  // the first pass ran at load, the last runs at the store
      fft_passes_ct_to<C, (MC > 0 ? MC : 2), 1, NPS - 1, R0>(row, Wy, !fwd, lane);
    else if constexpr (fuse1)
      fft_passes_ct<C, (MC > 0 ? MC : 2), 1, R0>(row, Wy, !fwd, lane);  // the first pass ran at load
    else if constexpr (MC > 0)
      fft_warp_ct<C, MC>(row, Wy, !fwd, lane);
    else
      fft_warp<C, DPT, POW2>(row, pl, Wy, !fwd, lane);
  }
  __syncthreads();
  const T sc = fwd ? (T)g.scaley : (T)1;
  if constexpr (fuseL) {
    if (!colok) return;
    const bool tr = iit < g.nxh;  // the x-Nyquist column holds raw values
    const C* ra = A + tb * RSY;
    const C* rb = A2 + tb * RSY;
    C* o0 = (C*)(jb.dst + fidx<T>(g, 2 * iit, 0, k));
    const size_t ys = (size_t)g.nxpp / 2;  // one y row, in complex values
#pragma unroll 1
    for (int mb = 0; mb < NSL / JS; ++mb) {
      const int j = tj + JS * mb;  // butterfly of the last pass (Ns = NSL, step 1)
      C va[RL], vb[RL];
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        va[r] = ra[fpad(j + r * NSL)];
        if (two) vb[r] = rb[fpad(j + r * NSL)];
      }
      if (tr) {
#pragma unroll
        for (int r = 1; r < RL; ++r) {
          C tw = Wy[r * j];
          if (!fwd) tw.y = -tw.y;
          va[r] = cmul(va[r], tw);
          if (two) vb[r] = cmul(vb[r], tw);
        }
        dft_reg<C, RL>(va, !fwd);
        if (two) dft_reg<C, RL>(vb, !fwd);
      }
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        const int y = j + r * NSL;
        C o = cmk<C>(va[r].x * sc, va[r].y * sc);
        if (two) {
          const C w2 = cmk<C>(vb[r].x * sc, vb[r].y * sc);
          const T ky = (T)g.yw[y];
          o = cmk<C>(o.x - ky * w2.y, o.y + ky * w2.x);
        }
        o0[(size_t)y * ys] = o;
      }
    }
    return;
  }
  if (colok) {
    const C* d = A + tb * RSY + fpad(tj);
    C* o1 = (C*)(jb.dst + fidx<T>(g, 2 * iit, tj, k));
    for (int j = tj; j < ny; j += JS) {
      const C v = *d;
      C o = cmk<C>(v.x * sc, v.y * sc);
      if (two) {
        const C v2 = d[TX * RSY];
        const C w2 = cmk<C>(v2.x * sc, v2.y * sc);
        const T ky = (T)g.yw[j];
        o = cmk<C>(o.x - ky * w2.y, o.y + ky * w2.x);
      }
      *o1 = o;
      d += JS + JS / 16;
      o1 = (C*)((T*)o1 + gstep);
    }
  }
}

// ===========================================================================
// x transforms of rows.  Real length nx = 2M through complex length M.
// ===========================================================================
template <typename C, typename T>
__device__ __forceinline__ void xinv_prep(const T* __restrict__ row, C* Z, int M, const C* __restrict__ Wn, int mulkx,
                                          T kxstep, int t0, int nthr) {
  // row: nxhp complex (interleaved); optional multiply by i*kx (kx = m*kxstep)
  for (int k = t0; k < M; k += nthr) {
    C Xk = cmk<C>(row[2 * k], row[2 * k + 1]);
    C Xm = cmk<C>(row[2 * (M - k)], row[2 * (M - k) + 1]);
    if (mulkx) {
      T a = kxstep * (T)k, b = kxstep * (T)(M - k);
      Xk = cmk<C>(-(a * Xk.y), a * Xk.x);
      Xm = cmk<C>(-(b * Xm.y), b * Xm.x);
    }
    if (k == 0) {
      Xk.y = 0;
      Xm.y = 0;
    }
    C s = cadd(Xk, cconj(Xm));
    C d = csub(Xk, cconj(Xm));
    C w = Wn[k];  // exp(-2 pi i k/N); need i*conj(w)*d
    C wc = cconj(w);
    C t = cmul(wc, d);
    Z[k] = cmk<C>(s.x - t.y, s.y + t.x);
  }
}

// forward post: Z = FFT_M(z) -> X_k k=0..M (scaled by 1/N)
template <typename C>
__device__ __forceinline__ C xfwd_post(const C* Z, int k, int M, const C* __restrict__ Wn, decltype(C().x) invN) {
  typedef decltype(C().x) T;
  if (k == 0) return cmk<C>((Z[0].x + Z[0].y) * invN, (T)0);
  if (k == M) return cmk<C>((Z[0].x - Z[0].y) * invN, (T)0);
  C a = Z[k], b = cconj(Z[M - k]);
  C e = cmk<C>((T)0.5 * (a.x + b.x), (T)0.5 * (a.y + b.y));
  C dd = csub(a, b);
  C o = cmk<C>((T)0.5 * dd.y, (T)-0.5 * dd.x);  // (a-b)/(2i)
  C w = Wn[k];
  C wo = cmul(w, o);
  return cmk<C>((e.x + wo.x) * invN, (e.y + wo.y) * invN);
}

// Parameters of the fused NL row kernel.
template <typename T>
struct NLArgs {
  const T* in[12];  // (kx,y): u v w t | dy u v w t | dz u v w t
  T* out[11];       // (kx,y): Au Av Aw At | uv vv vw vt | uw ww wt
  double coef_buoy; // N^2 / rhograd
  double rg;        // rhograd
  double tau_pen[IW_MAX_SUBD];  // 0.5/omega*(2/zh)
  int forcing;
  double f_xk, f_xm, f_om, f_t, f_amp_u, f_amp_w, f_amp_r;  // paddle
  double dx;
};

// In-place pre-pass of the inverse real transform for the pair (kk, M-kk) of a
// padded row holding X_0..X_M: Z_k = (X_k + conj X_{M-k}) + i conj(W_k) (X_k - conj X_{M-k}),
// after the optional multiplication by i kx.  0 <= kk <= M/2.
template <typename C, typename T>
__device__ __forceinline__ void xprep_pair(C* row, int kk, int M, const C* __restrict__ Wn, bool mulkx, T kxstep) {
  const int km = M - kk;
  const C X0 = row[fpad(kk)], X1 = row[fpad(km)];
  auto zk = [&](C Xk, C Xm, int k) {
    if (mulkx) {
      const T a = kxstep * (T)k, b = kxstep * (T)(M - k);
      Xk = cmk<C>(-(a * Xk.y), a * Xk.x);
      Xm = cmk<C>(-(b * Xm.y), b * Xm.x);
    }
    if (k == 0) {
      Xk.y = 0;
      Xm.y = 0;
    }
    const C s = cadd(Xk, cconj(Xm));
    const C d = csub(Xk, cconj(Xm));
    const C t = cmul(cconj(Wn[k]), d);
    return cmk<C>(s.x - t.y, s.y + t.x);
  };
  const C z0 = zk(X0, X1, kk);
  if (kk > 0 && kk < km) row[fpad(km)] = zk(X1, X0, km);
  row[fpad(kk)] = z0;
}

// forward post on a padded row: Z = FFT_M(z) -> X_k, k = 0..M (scaled by 1/N)
template <typename C>
__device__ __forceinline__ C xfwd_post_p(const C* row, int k, int M, const C* __restrict__ Wn,
                                         decltype(C().x) invN) {
  typedef decltype(C().x) T;
  if (k == 0 || k == M) {
    const C z = row[0];
    return k == 0 ? cmk<C>((z.x + z.y) * invN, (T)0) : cmk<C>((z.x - z.y) * invN, (T)0);
  }
  const C a = row[fpad(k)], b = cconj(row[fpad(M - k)]);
  const C e = cmk<C>((T)0.5 * (a.x + b.x), (T)0.5 * (a.y + b.y));
  const C dd = csub(a, b);
  const C o = cmk<C>((T)0.5 * dd.y, (T)-0.5 * dd.x);  // (a-b)/(2i)
  const C wo = cmul(Wn[k], o);
  return cmk<C>((e.x + wo.x) * invN, (e.y + wo.y) * invN);
}

// slots per padded x row (M+1 half-complex values)
__host__ __device__ __forceinline__ int xstride(int M) { return fpadlen(M + 1); }

// K_C: CTA per (j,k) row; 20 padded rows of M+1 values in shared memory; each
// warp transforms whole rows in place.
template <typename T, int DPT, bool POW2, int MC = 0>
__global__ void __launch_bounds__(256, (FftOcc<T, DPT>::v)) k_xrow_nl(Geo g, NLArgs<T> a, FftPlan pl,
                                                 const typename cplx_t<T>::type* __restrict__ Wm,
                                                 const typename cplx_t<T>::type* __restrict__ Wn) {
  typedef typename cplx_t<T>::type C;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int M = MC > 0 ? MC : g.nx / 2;  // a constant with a compile-time plan
  const int RS = xstride(M);
  C* buf = (C*)smraw;
  const int j = blockIdx.x, k = blockIdx.y;
  const int N = g.N;
  const int kl = k % N, ks = k / N;
  const bool nb_lo = (kl == 0 && k > 0);
  const bool nb_hi = (kl == N - 1 && k < g.nz - 1);
  const int knb = nb_lo ? k - 1 : k + 1;
  const int nrow = 16 + ((nb_lo || nb_hi) ? 4 : 0);
  const T kxs = (T)g.xw[1];
  const int tid = threadIdx.x, nthr = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = nthr >> 5;
  // rows 0..3 u v w t, 4..7 dx, 8..11 dy, 12..15 dz, 16..19 neighbour u v w t:
  // half-complex rows (M+1 values), all copies in flight at once
  // Element offsets of this (j, k) row and of the neighbour's, once per CTA.
  // A thread keeps its kk and walks the rows (fixed strides, no index
  // arithmetic per copy); kk = M, the last value of a row, goes to thread r.
  const size_t roff = fidx<T>(g, 0, j, k), roffn = fidx<T>(g, 0, j, knb);
  auto rsrc = [&](int r) -> const C* {
    return (const C*)((r < 4 ? a.in[r] : r < 16 ? a.in[r - 4] : a.in[r - 16]) + (r < 16 ? roff : roffn));
  };
  for (int kk = tid; kk < M; kk += nthr) {
    C* d = buf + fpad(kk);
#pragma unroll
    for (int r = 0; r < 20; ++r)
      if (r < nrow) cp_async_c<C>(d + r * RS, rsrc(r) + kk);
  }
  if (tid < nrow) cp_async_c<C>(buf + tid * RS + fpad(M), rsrc(tid) + M);
  cp_async_wait_all();
  __syncthreads();
  const int nh = M / 2 + 1;
  const int H2 = M / 2;
  if (MC > 0 && nthr % H2 == 0) {
    // a thread keeps its pair kk < M/2 and steps over rows by nthr/(M/2);
    // the middle pair kk = M/2 goes to thread r
    const int kk = tid % H2, rs = nthr / H2;
    for (int r = tid / H2; r < nrow; r += rs) xprep_pair<C, T>(buf + r * RS, kk, M, Wn, r >= 4 && r < 8, kxs);
    if (tid < nrow) xprep_pair<C, T>(buf + tid * RS, H2, M, Wn, tid >= 4 && tid < 8, kxs);
  } else {
    for (int q = tid; q < nrow * nh; q += nthr) {
      const int r = q / nh, kk = q - r * nh;
      xprep_pair<C, T>(buf + r * RS, kk, M, Wn, r >= 4 && r < 8, kxs);
    }
  }
  __syncthreads();
  for (int r = wid; r < nrow; r += nw) {
    if constexpr (MC > 0)
      fft_warp_ct<C, MC>(buf + r * RS, Wm, true, lane);
    else
      fft_warp<C, DPT, POW2>(buf + r * RS, pl, Wm, true, lane);
  }
  __syncthreads();
  // physical value i of row r
  auto P = [&](int r, int i) -> T& { return ((T*)(buf + r * RS))[2 * fpad(i >> 1) + (i & 1)]; };
  const int nx = 2 * M;
  // upwind interface penalty (solver.f:700-839); products overwrite rows 0..12
  for (int i = tid; i < nx; i += nthr) {
    const T u = P(0, i), v = P(1, i), w = P(2, i), t = P(3, i);
    const T ux = P(4, i), vx = P(5, i), wx = P(6, i);
    const T uy = P(8, i), vy = P(9, i), wy = P(10, i);
    const T uz = P(12, i), vz = P(13, i), wz = P(14, i);
    T qu = (T)-0.5 * (u * ux + v * uy + w * uz);
    T qv = (T)-0.5 * (u * vx + v * vy + w * vz);
    T qw = (T)-0.5 * (u * wx + v * wy + w * wz) + (T)a.coef_buoy * t;
    T qt = -(w * (T)a.rg);
    if (nb_lo && w > (T)0) {  // bottom point of subdomain ks: inflow from below
      const T tau = (T)a.tau_pen[ks], al = w;
      qu -= tau * (al * u - al * P(16, i));
      qv -= tau * (al * v - al * P(17, i));
      qw -= tau * (al * w - al * P(18, i));
      qt -= tau * (al * t - al * P(19, i));
    }
    if (nb_hi && w < (T)0) {
      const T tau = (T)a.tau_pen[ks], ga = -w;
      qu -= tau * (ga * u - ga * P(16, i));
      qv -= tau * (ga * v - ga * P(17, i));
      qw -= tau * (ga * w - ga * P(18, i));
      qt -= tau * (ga * t - ga * P(19, i));
    }
    if (a.forcing == IW_PADDLE_ALL_LEVELS || (a.forcing == IW_PADDLE_ABOVE_BOTTOM && k > 0)) {
      double xx = (double)i * a.dx, zz = g.zg[k];
      double arg = a.f_xk * xx - a.f_om * a.f_t;
      double sf, cf;
      sincos(arg, &sf, &cf);
      double czm = cos(a.f_xm * zz), szm = sin(a.f_xm * zz);
      qu += (T)(a.f_amp_u * czm * sf);
      qw += (T)(a.f_amp_w * szm * cf);
      qt += (T)(a.f_amp_r * szm * sf);
    }
    // 13 rows to transform: Qu Qv Qw Qt | uu uv uw ut | vv vw vt | ww wt
    P(0, i) = qu;
    P(1, i) = qv;
    P(2, i) = qw;
    P(3, i) = qt;
    P(4, i) = (T)-0.5 * u * u;
    P(5, i) = (T)-0.5 * u * v;
    P(6, i) = (T)-0.5 * u * w;
    P(7, i) = -(u * t);
    P(8, i) = (T)-0.5 * v * v;
    P(9, i) = (T)-0.5 * v * w;
    P(10, i) = -(v * t);
    P(11, i) = (T)-0.5 * w * w;
    P(12, i) = -(w * t);
  }
  __syncthreads();
  for (int r = wid; r < 13; r += nw) {
    if constexpr (MC > 0)
      fft_warp_ct<C, MC>(buf + r * RS, Wm, false, lane);
    else
      fft_warp<C, DPT, POW2>(buf + r * RS, pl, Wm, false, lane);
  }
  __syncthreads();
  const T invN = (T)1 / (T)nx;
  // outputs: A_q = X(Q_q) + i kx X(P_uq) for q = u v w t ; then uv vv vw vt uw ww wt
  // a thread keeps its kk and writes it in all 11 output rows; kk = M goes
  // to thread o
  auto outv = [&](int o, int kk) -> C {
    if (o < 4) {
      const C x1 = xfwd_post_p<C>(buf + o * RS, kk, M, Wn, invN);
      const C x2 = xfwd_post_p<C>(buf + (4 + o) * RS, kk, M, Wn, invN);
      const T kx = kxs * (T)kk;
      return cmk<C>(x1.x - kx * x2.y, x1.y + kx * x2.x);
    }
    // map: 4->uv(5) 5->vv(8) 6->vw(9) 7->vt(10) 8->uw(6) 9->ww(11) 10->wt(12)
    const int sr = o == 4 ? 5 : o == 5 ? 8 : o == 6 ? 9 : o == 7 ? 10 : o == 8 ? 6 : o == 9 ? 11 : 12;
    return xfwd_post_p<C>(buf + sr * RS, kk, M, Wn, invN);
  };
  for (int kk = tid; kk < M; kk += nthr) {
#pragma unroll 1
    for (int o = 0; o < 11; ++o) *((C*)(a.out[o] + roff) + kk) = outv(o, kk);
  }
  if (tid < 11) *((C*)(a.out[tid] + roff) + M) = outv(tid, M);
}

// ===========================================================================
// K_E: per (field q, real x index i, y index j, subdomain ks):
//   S    = B + (2/h) D Z                     (NL term at level n, spectral)
//   wnl  = fac1 S + fac2 Sn + fac3 Snm at the walls (w only, solver.f:267-284)
//   F2   = P(F1)                             (end-of-rhsfm round trip)
//   F*   = dt (fac1 S + fac2 Sn + fac3 Snm) + bdf1 F2 + bdf2 Fn + bdf3 Fnm
//   Snm <- S (becomes Sn), Fnm <- F2 (becomes Fn)      (solver.f:447-478)
//   F   <- cf(ii,j) * L F* per subdomain    (filter_3dlegenfourier)
// ===========================================================================
struct Coefs {
  double fac1, fac2, fac3, bdf1, bdf2, bdf3, bdfv, dt;
};

// u* = dt (extrapolated NL) + bdf1 F2 + bdf2 Fn + bdf3 Fnm, combined in FP64
// whatever the storage type: in FP32 the rounded coefficients (1/3) would
// make bdf1 + bdf2 + bdf3 differ from bdfv and bias every step the same way.
template <typename T>
__device__ __forceinline__ T bdf_combine(const Coefs& c, T se, T F2, T fn, T fnm) {
  return (T)(c.dt * (double)se + c.bdf1 * (double)F2 + c.bdf2 * (double)fn + c.bdf3 * (double)fnm);
}
// the same with every rounding written out
template <typename T>
__device__ __forceinline__ T bdf_combine_rn(const Coefs& c, T se, T F2, T fn, T fnm) {
  return (T)__fma_rn(c.bdf3, (double)fnm,
                     __fma_rn(c.bdf2, (double)fn, __fma_rn(c.bdf1, (double)F2, __dmul_rn(c.dt, (double)se))));
}


// one point of K_E: S = B + fac (D Z), u* from the BDF combination of the
// extrapolated S
template <typename T>
__device__ __forceinline__ void stageE_point(const Coefs& c, T fac, T f1, T f2, T f3, T b, T dz, T sn, T snm, T F2,
                                             T fn, T fnm, T& S, T& fsv) {
  S = fma_t(dz, fac, b);
  const T se = fma_t(f3, snm, fma_t(f2, sn, mul_t(f1, S)));
  fsv = bdf_combine_rn<T>(c, se, F2, fn, fnm);
}
// the extrapolated S in FP64 at the walls (the wall data of w)
template <typename T>
__device__ __forceinline__ double stageE_wall(T f1, T f2, T f3, T S, T sn, T snm) {
  return __fma_rn((double)f3, (double)snm, __fma_rn((double)f2, (double)sn, __dmul_rn((double)f1, (double)S)));
}
// the filtered value: cf (L f) = g + (cf - 1) g with g = f + (L - I) f
__device__ __forceinline__ double stageE_filtered(double f, double lf, double cfm1) {
  const double gv = __dadd_rn(f, lf);
  return __fma_rn(cfm1, gv, gv);
}

template <typename T>
struct EArgs {
  const T* B[4];
  const T* Z[4];
  const T* F1[4];
  const T* Fn[4];
  const T* Snold[4];
  T* Snm_w[4];  // in: S_{n-2}; out: S (new level n-1 after rotation)
  T* Fnm_w[4];  // in: F_{n-2}; out: F2 (new level n-1)
  T* F[4];      // out: filtered u*
  double* wnl;  // (nxpp,ny,2)
  int filter;
  // k_stageE_b: its zero-padded operators as one table built once on the
  // host ([NM][NP] doubles of L - I, then [NM][NP] T of D, the size rounded
  // up to 16 bytes); null: every CTA builds them from D and the filter
  const void* ops;
  unsigned ops_bytes;
};

template <typename T>
__device__ __forceinline__ void stageE_tile(const Geo& g, const EArgs<T>& a, const Coefs& c) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int N = g.N;
  double* sL = (double*)smraw;  // N*N, L - I in FP64 (see below)
  T* sD = (T*)(sL + N * N);     // N*N
  T* tz = sD + N * N;           // N*kTX: Z tile
  T* tf = tz + N * kTX;         // N*kTX: F* tile
  for (int t = threadIdx.x; t < N * N; t += blockDim.x) {
    sD[t] = (T)g.D[t];
    sL[t] = g.Lfil[t] - (t / N == t % N ? 1.0 : 0.0);
  }
  const int q = blockIdx.z;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i = blockIdx.x * kTX + lane;
  const int j = blockIdx.y % g.ny, ks = blockIdx.y / g.ny;
  const bool act = i < g.nxpp;
  for (int k = w; k < N; k += kTW) tz[k * kTX + lane] = act ? a.Z[q][fidx<T>(g, i, j, ks * N + k)] : (T)0;
  __syncthreads();
  const T fac = (T)g.hfac[ks];
  const T f1 = (T)c.fac1, f2 = (T)c.fac2, f3 = (T)c.fac3;
  for (int k1 = w; k1 < N; k1 += kTW) {
    T fsv = 0;
    if (act) {
      const int kk = ks * N + k1;
      const size_t p = fidx<T>(g, i, j, kk);
      const T* dr = sD + k1 * N;
      T s = 0;
#pragma unroll 4
      for (int k2 = 0; k2 < N; ++k2) s += dr[k2] * tz[k2 * kTX + lane];
      const T S = a.B[q][p] + s * fac;
      const T sn = a.Snold[q][p];
      const T snm = a.Snm_w[q][p];
      if (q == 2 && ((kk == 0) || (kk == g.nz - 1))) {
        const int side = kk == 0 ? 0 : 1;
        a.wnl[(size_t)i + (size_t)g.nxpp * ((size_t)j + (size_t)g.ny * side)] =
            (double)f1 * (double)S + (double)f2 * (double)sn + (double)f3 * (double)snm;
      }
      const T se = f1 * S + f2 * sn + f3 * snm;
      const T F2 = proj_val<T>(g, a.F1[q], i, j, kk);
      const T fn = a.Fn[q][p];
      const T fnm = a.Fnm_w[q][p];
      fsv = bdf_combine<T>(c, se, F2, fn, fnm);
      a.Snm_w[q][p] = S;
      a.Fnm_w[q][p] = F2;
    }
    tf[k1 * kTX + lane] = fsv;
  }
  __syncthreads();
  if (!act) return;
  // The Legendre filter acts on the state itself every step: L - I has O(1)
  // entries (a projector onto the damped modes), so FP32 entries would add
  // the same rounding error to the state each step.  It runs in FP64 with
  // one rounding of the result; cf - 1 is small for the energetic modes.
  const double cfm1 = a.filter ? g.cfour[(size_t)j * g.nxhp + (i >> 1)] - 1.0 : 0.0;
  for (int k1 = w; k1 < N; k1 += kTW) {
    T o;
    if (a.filter) {
      const double* lr = sL + k1 * N;
      double s = 0;
#pragma unroll 4
      for (int k2 = 0; k2 < N; ++k2) s += lr[k2] * (double)tf[k2 * kTX + lane];
      const double gv = (double)tf[k1 * kTX + lane] + s;  // L f = f + (L - I) f
      o = (T)(gv + cfm1 * gv);                            // cf g = g + (cf - 1) g
    } else {
      o = tf[k1 * kTX + lane];
    }
    a.F[q][fidx<T>(g, i, j, ks * N + k1)] = o;
  }
}

// Tiled K_E with its input tiles staged by bulk asynchronous copies and the
// z operators unrolled at a compile-time size NM >= N (the zero-padded
// bucket of the register-column kernels).  The CTA tiling is stageE_tile's
// (32 x points of one (y, subdomain), 8 warps) and so are the sums, in the
// same order (every rounding written out, so it agrees to rounding).  The
// seven input tiles (Z, B, S_n, S_{n-1}, F1, F_n, F_{n-1}) are requested at
// once, one cp.async.bulk per row completing on an mbarrier (Z on its own,
// so that D Z starts while the rest lands).  Warp w computes all of its
// output rows k1 = w + 8 r at once, so each column value feeds every row and
// each pair of operator entries is one 8-byte broadcast; with NM known every
// shared-memory address is a base plus an immediate.  A row of 32 points is
// copied from the 16-byte boundary at or below its first point (FP32 rows of
// an nxpp = 2 (mod 4) field start 8 bytes into a unit); the copy may run up to
// 15 bytes past the field's end, inside the 16 bytes every field buffer is
// allocated with beyond its end.  The launch requires nxpp*ny*sizeof(T) to be
// a multiple of 16, so that every row of a CTA has the same offset.
// z operators of the register-column kernels and of k_stageE_b<.., true>: kernel
// parameters, i.e. served from the constant bank
template <typename T, int NM>
struct ZOp {
  T D[NM * NM];       // D[k1*NM + k2], zero outside N x N
  double L[NM * NM];  // precombined Legendre filter minus the identity, same layout (FP64, see k_stageE)
};
constexpr int kEBArr = 7;
template <typename T>
__host__ __device__ inline int eb_rs() {  // tile row stride (elements): 32 points and room for the offset
  return kTX + 16 / (int)sizeof(T);
}
__host__ __device__ constexpr int eb_np(int NM) { return (NM + 1) & ~1; }  // operator row stride: pairs stay aligned
template <typename T>
__host__ inline size_t eb_smem(int N, int NM, bool cb = false) {
  return 16 + ((size_t)NM + (size_t)(kEBArr - 1) * N) * eb_rs<T>() * sizeof(T) +
         (cb ? 0 : (size_t)NM * eb_np(NM) * sizeof(double) + (size_t)NM * eb_np(NM) * sizeof(T)) +
         (size_t)NM * kTX * sizeof(T);
}
// two consecutive operator entries (an 8-byte broadcast load for FP32)
__device__ __forceinline__ void ld_pair(const float* p, float& a, float& b) {
  const float2 v = *(const float2*)p;
  a = v.x;
  b = v.y;
}
__device__ __forceinline__ void ld_pair(const double* p, double& a, double& b) {
  a = p[0];
  b = p[1];
}

// CB: D and L - I from the kernel parameter op (the constant bank; a warp's
// rows are warp-uniform, so every operator entry is a uniform load) instead of
// shared memory; the same sums in the same order.
template <typename T, int NM, bool CB = false>
__global__ void __launch_bounds__(kTX* kTW) k_stageE_b(Geo g, EArgs<T> a, Coefs c, int* __restrict__ err,
                                                       const __grid_constant__ ZOp<T, NM> op) {
  constexpr int NP = eb_np(NM), RB = (NM + kTW - 1) / kTW;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int N = g.N, RS = eb_rs<T>();
  uint64_t* bar = (uint64_t*)smraw;  // [0]: Z, [1]: the other six tiles
  T* tiles = (T*)(smraw + 16);       // Z: [NM][RS], then arrays 1..6: [N][RS] each
  double* sL = (double*)(tiles + ((size_t)NM + (size_t)(kEBArr - 1) * N) * RS);  // [NM][NP]: L - I (not CB)
  T* sD = (T*)(sL + (CB ? 0 : NM * NP));                                          // [NM][NP] (not CB)
  T* tf = sD + (CB ? 0 : NM * NP);                                                // [NM][kTX]: F* tile
  const int q = blockIdx.z;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int i0 = blockIdx.x * kTX, i = i0 + lane;
  const int j = blockIdx.y % g.ny, ks = blockIdx.y / g.ny;
  const int nval = min(kTX, g.nxpp - i0);
  const bool pre = !CB && a.ops != nullptr;
  if (tid == 0) {
    mbar_init(&bar[0], (uint32_t)N + (pre ? 1u : 0u));
    mbar_init(&bar[1], (uint32_t)((kEBArr - 1) * N));
  }
  __syncthreads();
  if (pre && tid == (int)blockDim.x - 1) {  // the operators, with the Z tile (the copy may run 15 bytes into tf)
    mbar_expect_tx(&bar[0], a.ops_bytes);
    bulk_g2s(sL, a.ops, a.ops_bytes, &bar[0]);
  }
  for (int t = tid; t < kEBArr * N; t += blockDim.x) {
    const int arr = t / N, k = t - arr * N;
    const T* base = arr == 0 ? a.Z[q]
                    : arr == 1 ? a.B[q]
                    : arr == 2 ? a.Snold[q]
                    : arr == 3 ? a.Snm_w[q]
                    : arr == 4 ? a.F1[q]
                    : arr == 5 ? a.Fn[q]
                               : a.Fnm_w[q];
    const uintptr_t ga = (uintptr_t)(base + fidx<T>(g, i0, j, ks * N + k));
    const uint32_t off = (uint32_t)(ga & 15u);
    const uint32_t bytes = (off + (uint32_t)nval * (uint32_t)sizeof(T) + 15u) & ~15u;
    uint64_t* b = &bar[arr == 0 ? 0 : 1];
    T* dst = tiles + (arr == 0 ? (size_t)k : (size_t)NM + (size_t)(arr - 1) * N + k) * RS;
    mbar_expect_tx(b, bytes);
    bulk_g2s(dst, (const void*)(ga - off), bytes, b);
  }
  // operators zero-padded to NM x NM (unless copied above), the padding rows of
  // the Z and F* tiles zero
  if (!pre && !CB) {
    for (int t = tid; t < NM * NP; t += blockDim.x) {
      const int r = t / NP, cc = t - r * NP;
      const bool in = r < N && cc < N;
      sD[t] = in ? (T)g.D[r * N + cc] : (T)0;
      sL[t] = in ? g.Lfil[r * N + cc] - (r == cc ? 1.0 : 0.0) : 0.0;
    }
  }
  for (int t = N * RS + tid; t < NM * RS; t += blockDim.x) tiles[t] = (T)0;
  for (int t = N * kTX + tid; t < NM * kTX; t += blockDim.x) tf[t] = (T)0;
  // element offset of this CTA's first point inside each copied row (the
  // same for every row: the planes are whole 16-byte units)
  const int eo = (int)((((size_t)i0 + (size_t)g.nxpp * ((size_t)j + (size_t)g.ny * (size_t)(ks * N))) * sizeof(T)) &
                       15u) /
                 (int)sizeof(T);
  const bool ok0 = mbar_wait(&bar[0], 0, 2000000000ull);
  __syncthreads();  // the operator tables and padding are in place
  const bool act = i < g.nxpp;
  const T fac = (T)g.hfac[ks];
  const T f1 = (T)c.fac1, f2 = (T)c.fac2, f3 = (T)c.fac3;
  // D Z for this warp's rows; lanes past the field's end compute on stale
  // tile entries and store nothing
  T dz[RB];
#pragma unroll
  for (int r = 0; r < RB; ++r) dz[r] = 0;
  const T* zc = tiles + eo + lane;  // this lane's column of the Z tile
  const T* dw = sD + w * NP;        // row w of D; row w + 8 r is dw + 8 r NP
#pragma unroll
  for (int k2 = 0; k2 < NM; k2 += 2) {
    const T z0 = zc[k2 * RS];
    const T z1 = k2 + 1 < NM ? zc[(k2 + 1) * RS] : (T)0;
#pragma unroll
    for (int r = 0; r < RB; ++r) {
      if (r < RB - 1 || w + kTW * r < NM) {
        T d0, d1;
        if constexpr (CB) {
          const T* od = op.D + (w + kTW * r) * NM + k2;
          if (k2 + 1 < NM) {
            d0 = od[0];
            d1 = od[1];
            dz[r] = fma_t(d1, z1, fma_t(d0, z0, dz[r]));
          } else {
            dz[r] = fma_t(od[0], z0, dz[r]);
          }
        } else if (k2 + 1 < NM) {
          ld_pair(dw + r * kTW * NP + k2, d0, d1);
          dz[r] = fma_t(d1, z1, fma_t(d0, z0, dz[r]));
        } else {
          dz[r] = fma_t(dw[r * kTW * NP + k2], z0, dz[r]);
        }
      }
    }
  }
  const bool ok1 = mbar_wait(&bar[1], 0, 2000000000ull);
  if (__syncthreads_or(!(ok0 && ok1))) {  // a copy never completed: report, let the copies finish, leave
    if (tid == 0) err[1] = 1;
    mbar_wait(&bar[0], 0, 2000000000ull);
    mbar_wait(&bar[1], 0, 2000000000ull);
    return;
  }
#pragma unroll
  for (int r = 0; r < RB; ++r) {
    const int k1 = w + kTW * r;
    if (k1 >= N) break;
    T fsv = 0;
    if (act) {
      const int kk = ks * N + k1;
      const size_t p = fidx<T>(g, i, j, kk);
      const size_t e = (size_t)NM * RS + (size_t)k1 * RS + eo + lane;  // array 1 (B), row k1
      const size_t AS = (size_t)N * RS;
      const T sn = tiles[e + 1 * AS];
      const T snm = tiles[e + 2 * AS];
      T F2;
      if (i < 2) {
        const T va = tiles[e + 3 * AS];
        const T vb = a.F1[q][fidx<T>(g, i, (g.ny - j) % g.ny, kk)];
        F2 = i == 0 ? (T)0.5 * (va + vb) : (T)0.5 * (va - vb);
      } else if (i >= g.nx) {
        F2 = i == g.nx ? tiles[e + 3 * AS] * (T)g.scaley : (T)0;
      } else {
        F2 = tiles[e + 3 * AS];
      }
      const T fn = tiles[e + 4 * AS];
      const T fnm = tiles[e + 5 * AS];
      T S;
      stageE_point<T>(c, fac, f1, f2, f3, tiles[e], dz[r], sn, snm, F2, fn, fnm, S, fsv);
      if (q == 2 && ((kk == 0) || (kk == g.nz - 1))) {
        const int side = kk == 0 ? 0 : 1;
        a.wnl[(size_t)i + (size_t)g.nxpp * ((size_t)j + (size_t)g.ny * side)] = stageE_wall<T>(f1, f2, f3, S, sn, snm);
      }
      a.Snm_w[q][p] = S;
      a.Fnm_w[q][p] = F2;
    }
    tf[k1 * kTX + lane] = fsv;
  }
  __syncthreads();
  if (!act) return;
  if (!a.filter) {
#pragma unroll
    for (int r = 0; r < RB; ++r) {
      const int k1 = w + kTW * r;
      if (k1 < N) a.F[q][fidx<T>(g, i, j, ks * N + k1)] = tf[k1 * kTX + lane];
    }
    return;
  }
  const double cfm1 = g.cfour[(size_t)j * g.nxhp + (i >> 1)] - 1.0;
  // (L - I) F* in FP64 for all of this warp's rows at once, sums in k2 order
  double s2[RB];
#pragma unroll
  for (int r = 0; r < RB; ++r) s2[r] = 0.0;
  const double* lw = sL + w * NP;
#pragma unroll
  for (int k2 = 0; k2 < NM; ++k2) {
    const double f = (double)tf[k2 * kTX + lane];
#pragma unroll
    for (int r = 0; r < RB; ++r)
      if (r < RB - 1 || w + kTW * r < NM)
        s2[r] = __fma_rn(CB ? op.L[(w + kTW * r) * NM + k2] : lw[r * kTW * NP + k2], f, s2[r]);
  }
#pragma unroll
  for (int r = 0; r < RB; ++r) {
    const int k1 = w + kTW * r;
    if (k1 < N) a.F[q][fidx<T>(g, i, j, ks * N + k1)] = (T)stageE_filtered((double)tf[k1 * kTX + lane], s2[r], cfm1);
  }
}

// The tiled K_E kernels.  FP32 fields: at most 32 registers so that 8 CTAs
// fit on an SM (the kernel waits on global loads, more resident warps pay);
// FP64 fields: the compiler's own allocation.
template <typename T>
__global__ void __launch_bounds__(kTX* kTW) k_stageE(Geo g, EArgs<T> a, Coefs c) {
  stageE_tile<T>(g, a, c);
}
__global__ void __launch_bounds__(kTX* kTW, 8) k_stageE_f32(Geo g, EArgs<float> a, Coefs c) {
  stageE_tile<float>(g, a, c);
}

// ---------------------------------------------------------------------------
// Register-column variants of K_A and K_E for N <= 33.  A thread owns one
// (x, y) point of one subdomain and keeps its N values of the column in
// registers; thread t addresses element t of every z-plane, so each warp
// reads and writes 128-byte contiguous runs.  The N x N operators (D and the
// precombined filter minus the identity, zero-padded to NM x NM; a filter
// close to the identity is applied as f + (L - I) f so that rounding its
// entries does not bias every step) are kernel parameters, i.e. they
// sit in the constant bank, and the fully unrolled products take them as
// immediate operands: about one instruction per multiply-add.
// ---------------------------------------------------------------------------

template <typename T, int NM>
__global__ void __launch_bounds__(128) k_stageA_r(Geo g, const __grid_constant__ ZOp<T, NM> op,
                                                   const T* __restrict__ F0, const T* __restrict__ F1_,
                                                   const T* __restrict__ F2_, const T* __restrict__ F3_,
                                                   T* __restrict__ O0, T* __restrict__ O1, T* __restrict__ O2,
                                                   T* __restrict__ O3, T* __restrict__ Z0, T* __restrict__ Z1,
                                                   T* __restrict__ Z2, T* __restrict__ Z3, int proj,
                                                   int* __restrict__ err) {
  const int q = blockIdx.z, ks = blockIdx.y, N = g.N;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.plane) return;
  const int i = (int)(t % g.nxpp), j = (int)(t / g.nxpp);
  const T* F = q == 0 ? F0 : q == 1 ? F1_ : q == 2 ? F2_ : F3_;
  T* O = q == 0 ? O0 : q == 1 ? O1 : q == 2 ? O2 : O3;
  T* Z = q == 0 ? Z0 : q == 1 ? Z1 : q == 2 ? Z2 : Z3;
  const bool wzero = q == 2 && j == 0 && i < 2;  // wc(1,1,:) = 0, solver.f:66-69
  // the projection changes only the kx = 0 and Nyquist columns: every other
  // point is a plain copy, read and written with fixed plane strides
  const bool special = proj && (i < 2 || i >= g.nx);
  const size_t pl = g.plane, o0 = (size_t)(ks * N) * pl + t;
  T col[NM];
  bool bad = false;
  if (!special) {
#pragma unroll
    for (int k = 0; k < NM; ++k) {
      T x = 0;
      if (k < N) {
        x = F[o0 + (size_t)k * pl];
        bad |= !isfinite(x);
        if (wzero) x = (T)0;
        O[o0 + (size_t)k * pl] = x;
      }
      col[k] = x;
    }
  } else {
#pragma unroll
    for (int k = 0; k < NM; ++k) {
      T x = 0;
      if (k < N) {
        x = proj_val<T>(g, F, i, j, ks * N + k);
        bad |= !isfinite(x);
        if (wzero) x = (T)0;
        O[o0 + (size_t)k * pl] = x;
      }
      col[k] = x;
    }
  }
  if (bad) err[0] = 1;  // the state of the last step holds a NaN or Inf
  const T fac = (T)g.hfac[ks];
#pragma unroll
  for (int k1 = 0; k1 < NM; ++k1) {
    if (k1 < N) {
      T s = 0;
#pragma unroll
      for (int k2 = 0; k2 < NM; ++k2) s = fma_t(op.D[k1 * NM + k2], col[k2], s);
      Z[o0 + (size_t)k1 * pl] = mul_t(s, fac);
    }
  }
}

template <typename T, int NM>
__global__ void __launch_bounds__(128) k_stageE_r(Geo g, EArgs<T> a, Coefs c, const __grid_constant__ ZOp<T, NM> op) {
  const int q = blockIdx.z, ks = blockIdx.y, N = g.N;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.plane) return;
  const int i = (int)(t % g.nxpp), j = (int)(t / g.nxpp);
  T zc[NM];
#pragma unroll
  for (int k = 0; k < NM; ++k) zc[k] = k < N ? a.Z[q][(size_t)(ks * N + k) * g.plane + t] : (T)0;
  const T fac = (T)g.hfac[ks];
  const T f1 = (T)c.fac1, f2 = (T)c.fac2, f3 = (T)c.fac3;
  const T* Bq = a.B[q];
  const T* Snq = a.Snold[q];
  const T* F1q = a.F1[q];
  const T* Fnq = a.Fn[q];
  T* Snmq = a.Snm_w[q];
  T* Fnmq = a.Fnm_w[q];
  // Rolling window: the inputs of row k1+PF are loaded before the stores of
  // row k1, so the loads of several rows are in flight at once (the pointers
  // are not known to be distinct, so the compiler would not hoist them).
  constexpr int PF = 4;
  T wb[PF], wsn[PF], wsnm[PF], wf2[PF], wfn[PF], wfnm[PF];
#pragma unroll
  for (int k1 = 0; k1 < PF; ++k1) {
    if (k1 < N) {
      const int kk = ks * N + k1;
      const size_t p = (size_t)kk * g.plane + t;
      wb[k1] = Bq[p];
      wsn[k1] = Snq[p];
      wsnm[k1] = Snmq[p];
      wf2[k1] = proj_val<T>(g, F1q, i, j, kk);
      wfn[k1] = Fnq[p];
      wfnm[k1] = Fnmq[p];
    }
  }
  T fs[NM];
#pragma unroll
  for (int k1 = 0; k1 < NM; ++k1) {
    T fsv = 0;
    if (k1 < N) {
      const int sl = k1 % PF;
      const T b = wb[sl], sn = wsn[sl], snm = wsnm[sl], F2 = wf2[sl], fn = wfn[sl], fnm = wfnm[sl];
      if (k1 + PF < NM && k1 + PF < N) {
        const int kn = ks * N + k1 + PF;
        const size_t pn = (size_t)kn * g.plane + t;
        wb[sl] = Bq[pn];
        wsn[sl] = Snq[pn];
        wsnm[sl] = Snmq[pn];
        wf2[sl] = proj_val<T>(g, F1q, i, j, kn);
        wfn[sl] = Fnq[pn];
        wfnm[sl] = Fnmq[pn];
      }
      const int kk = ks * N + k1;
      const size_t p = (size_t)kk * g.plane + t;
      T s = 0;
#pragma unroll
      for (int k2 = 0; k2 < NM; ++k2) s += op.D[k1 * NM + k2] * zc[k2];
      const T S = b + s * fac;
      if (q == 2 && ((kk == 0) || (kk == g.nz - 1)))
        a.wnl[t + (kk == 0 ? 0 : g.plane)] = (double)f1 * (double)S + (double)f2 * (double)sn + (double)f3 * (double)snm;
      const T se = f1 * S + f2 * sn + f3 * snm;
      fsv = bdf_combine<T>(c, se, F2, fn, fnm);
      Snmq[p] = S;
      Fnmq[p] = F2;
    }
    fs[k1] = fsv;
  }
  const double cfm1 = a.filter ? g.cfour[(size_t)j * g.nxhp + (i >> 1)] - 1.0 : 0.0;
#pragma unroll
  for (int k1 = 0; k1 < NM; ++k1) {
    if (k1 < N) {
      T o;
      if (a.filter) {
        double s = 0;
#pragma unroll
        for (int k2 = 0; k2 < NM; ++k2) s += op.L[k1 * NM + k2] * (double)fs[k2];  // (L - I) f in FP64
        const double gv = (double)fs[k1] + s;
        o = (T)(gv + cfm1 * gv);
      } else {
        o = fs[k1];
      }
      a.F[q][(size_t)(ks * N + k1) * g.plane + t] = o;
    }
  }
}

// rotational viscous term at the walls (solver.f:318-394, rotvisc 1210-1253):
// wviscrot = -nu * (fac1 rot(n) + fac2 rot(n-1) + fac3 rot(n-2)),
// rot = (kx^2+ky^2) w + i kx du/dz + i ky dv/dz at k0.
template <typename T>
__global__ void k_wviscrot(Geo g, const T* __restrict__ u1, const T* __restrict__ v1, const T* __restrict__ w1,
                           const T* __restrict__ un, const T* __restrict__ vn, const T* __restrict__ wn,
                           const T* __restrict__ unm, const T* __restrict__ vnm, const T* __restrict__ wnm, Coefs c,
                           double xnu, double* __restrict__ wvr) {
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long total = (long)g.nxhp * g.ny * 2;
  if (gid >= total) return;
  int ii = gid % g.nxhp;
  long r = gid / g.nxhp;
  int j = r % g.ny;
  int side = r / g.ny;
  const int N = g.N;
  int ks = side == 0 ? 0 : g.ns - 1;
  int k0 = side == 0 ? 0 : N - 1;
  double fac = g.hfac[ks];
  double xw = g.xw[ii], yw = g.yw[j];
  double rr = 0, ri = 0;
  for (int l = 0; l < 3; ++l) {
    const T* U = l == 0 ? u1 : l == 1 ? un : unm;
    const T* V = l == 0 ? v1 : l == 1 ? vn : vnm;
    const T* W = l == 0 ? w1 : l == 1 ? wn : wnm;
    double dur = 0, dui = 0, dvr = 0, dvi = 0;
    for (int k2 = 0; k2 < N; ++k2) {
      int kk = ks * N + k2;
      double d = g.D[k0 * N + k2];
      double ur, ui, vr, vi;
      if (l == 0) {
        ur = proj_val<T>(g, U, 2 * ii, j, kk);
        ui = proj_val<T>(g, U, 2 * ii + 1, j, kk);
        vr = proj_val<T>(g, V, 2 * ii, j, kk);
        vi = proj_val<T>(g, V, 2 * ii + 1, j, kk);
      } else {
        ur = U[fidx<T>(g, 2 * ii, j, kk)];
        ui = U[fidx<T>(g, 2 * ii + 1, j, kk)];
        vr = V[fidx<T>(g, 2 * ii, j, kk)];
        vi = V[fidx<T>(g, 2 * ii + 1, j, kk)];
      }
      dur += d * ur;
      dui += d * ui;
      dvr += d * vr;
      dvi += d * vi;
    }
    dur *= fac;
    dui *= fac;
    dvr *= fac;
    dvi *= fac;
    int kk0 = ks * N + k0;
    double wr, wi;
    if (l == 0) {
      wr = proj_val<T>(g, W, 2 * ii, j, kk0);
      wi = proj_val<T>(g, W, 2 * ii + 1, j, kk0);
    } else {
      wr = W[fidx<T>(g, 2 * ii, j, kk0)];
      wi = W[fidx<T>(g, 2 * ii + 1, j, kk0)];
    }
    double re = xw * xw * wr + yw * yw * wr - xw * dui - yw * dvi;
    double im = xw * xw * wi + yw * yw * wi + xw * dur + yw * dvr;
    double f = l == 0 ? c.fac1 : l == 1 ? c.fac2 : c.fac3;
    rr += f * re;
    ri += f * im;
  }
  size_t base = (size_t)g.nxpp * ((size_t)j + (size_t)g.ny * side) + 2 * ii;
  wvr[base] = -(xnu * rr);
  wvr[base + 1] = -(xnu * ri);
}

// ===========================================================================
// Band factorisation (penalty.f:403-634 assembly, band_lu.f:19-34 packing,
// bandludcmp.f:238-440 SGBTF2).  One warp per system; the arithmetic follows
// the reference order with no fused multiply-add, so the factors equal the
// CPU ones bit for bit.
// ===========================================================================
struct SysDesc {
  double eps;
  double tau1_bot, tau2_top;  // for the RHS boundary rows
  int ifbcbot, ifbctop;
  int pad[2];
};

struct FactorArgs {
  const SysDesc* sys = nullptr;
  const double* pen = nullptr;  // per system: 6*ns (alpha,beta,gamma,delta,tau1,tau2)
  double* ab = nullptr;         // per system: ldab*nz
  int* ipiv = nullptr;          // per system: nz
  int* info = nullptr;          // per system
  int nsys = 0;
  const double* D = nullptr;
  const double* D2 = nullptr;
  const double* zh = nullptr;  // ns
  int assemble = 1;            // 0: ab already holds the packed matrix (bandlu_solve_)
  int factor = 1;              // 0: assemble only (block-inverse systems)
};

__device__ __forceinline__ double& ABr(double* ab, int ldab, int r, int c) {
  return ab[(size_t)(r - 1) + (size_t)ldab * (size_t)(c - 1)];
}

__global__ void k_factor(Geo g, FactorArgs fa) {
  const int warps = blockDim.x / 32;
  const int s = blockIdx.x * warps + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (s >= fa.nsys) return;
  const int n = g.nz, N = g.N, ns = g.ns, kl = N, ku = N, ldab = 2 * kl + ku + 1;
  double* ab = fa.ab + (size_t)s * ldab * n;
  int* ipiv = fa.ipiv + (size_t)s * n;
  const double eps = fa.sys[s].eps;
  const double* pen = fa.pen + (size_t)s * 6 * ns;
  const double *pa = pen, *pb = pen + ns, *pg = pen + 2 * ns, *pd = pen + 3 * ns, *pt1 = pen + 4 * ns,
               *pt2 = pen + 5 * ns;
  const double* d = fa.D;
  const double* d2 = fa.D2;
  if (fa.assemble) {
  // zero the band
  for (size_t t = lane; t < (size_t)ldab * n; t += 32) ab[t] = 0.0;
  __syncwarp();
  // A(r,c) 0-based -> band row kl+ku+1+r-c (1-based), column c+1
#define AEL(r, c) ABr(ab, ldab, kl + ku + 1 + (r) - (c), (c) + 1)
  for (int ks = 0; ks < ns; ++ks) {
    const double ybar = fa.zh[ks];
    const double ybarl = ks > 0 ? fa.zh[ks - 1] : 0.0;
    const double ybarr = ks < ns - 1 ? fa.zh[ks + 1] : 0.0;
    const int km = ks * N;
    const double h2 = rmul(2.0 / ybar, 2.0 / ybar);
    const double eh = rmul(eps, h2);
    for (int t = lane; t < N * N; t += 32) {
      int k1 = t / N, k2 = t % N;
      AEL(km + k1, km + k2) = -rmul(eh, d2[k1 * N + k2]);
    }
    __syncwarp();
    for (int k1 = lane; k1 < N; k1 += 32) AEL(km + k1, km + k1) = radd(AEL(km + k1, km + k1), 1.0);
    __syncwarp();
    if (lane == 0) AEL(km, km) = radd(AEL(km, km), rmul(pt1[ks], pa[ks]));
    __syncwarp();
    {
      double cf = -__ddiv_rn(rmul(rmul(rmul(pt1[ks], pb[ks]), eps), 2.0), ybar);
      for (int k = lane; k < N; k += 32) AEL(km, km + k) = radd(AEL(km, km + k), rmul(cf, d[0 * N + k]));
    }
    __syncwarp();
    if (lane == 0) AEL(km + N - 1, km + N - 1) = radd(AEL(km + N - 1, km + N - 1), rmul(pt2[ks], pg[ks]));
    __syncwarp();
    {
      double cf = __ddiv_rn(rmul(rmul(rmul(pt2[ks], pd[ks]), eps), 2.0), ybar);
      for (int k = lane; k < N; k += 32)
        AEL(km + N - 1, km + k) = radd(AEL(km + N - 1, km + k), rmul(cf, d[(N - 1) * N + k]));
    }
    __syncwarp();
    if (ns > 1 && ks != 0) {
      if (lane == 0) AEL(km, km) = rsub(AEL(km, km), rmul(rmul(0.5, pt1[ks]), pa[ks]));
      __syncwarp();
      double cf = __ddiv_rn(rmul(rmul(rmul(rmul(0.5, pt1[ks]), pb[ks]), eps), 2.0), ybar);
      for (int k = lane; k < N; k += 32) AEL(km, km + k) = radd(AEL(km, km + k), rmul(cf, d[0 * N + k]));
      __syncwarp();
      for (int k = lane; k < N; k += 32) AEL(km, km - N + k) = 0.0;
      __syncwarp();
      if (lane == 0) AEL(km, km - 1) = -rmul(rmul(0.5, pt1[ks]), pa[ks]);
      __syncwarp();
      cf = __ddiv_rn(rmul(rmul(rmul(rmul(0.5, pt1[ks]), pb[ks]), eps), 2.0), ybarl);
      for (int k = lane; k < N; k += 32)
        AEL(km, km - N + k) = radd(AEL(km, km - N + k), rmul(cf, d[(N - 1) * N + k]));
      __syncwarp();
    }
    if (ns > 1 && ks != ns - 1) {
      if (lane == 0) AEL(km + N - 1, km + N - 1) = rsub(AEL(km + N - 1, km + N - 1), rmul(rmul(0.5, pt2[ks]), pg[ks]));
      __syncwarp();
      double cf = -__ddiv_rn(rmul(rmul(rmul(rmul(0.5, pt2[ks]), pd[ks]), eps), 2.0), ybar);
      for (int k = lane; k < N; k += 32)
        AEL(km + N - 1, km + k) = radd(AEL(km + N - 1, km + k), rmul(cf, d[(N - 1) * N + k]));
      __syncwarp();
      // a(km+1, km+nzloc+k) = 0: outside the band for nzloc >= 2 except the
      // row's own band part, which is zero here already
      if (lane == 0) AEL(km + N - 1, km + N) = rsub(AEL(km + N - 1, km + N), rmul(rmul(0.5, pt2[ks]), pg[ks]));
      __syncwarp();
      cf = -__ddiv_rn(rmul(rmul(rmul(rmul(0.5, pt2[ks]), pd[ks]), eps), 2.0), ybarr);
      for (int k = lane; k < N; k += 32)
        AEL(km + N - 1, km + N + k) = radd(AEL(km + N - 1, km + N + k), rmul(cf, d[0 * N + k]));
      __syncwarp();
    }
  }
#undef AEL
  }
  if (!fa.factor) return;
  // SGBTF2
  const int kv = ku + kl;
  int info = 0;
  for (int jj = ku + 2; jj <= min(kv, n); ++jj)
    for (int i = kv - jj + 2 + lane; i <= kl; i += 32) ABr(ab, ldab, i, jj) = 0.0;
  __syncwarp();
  int ju = 1;
  for (int j = 1; j <= n; ++j) {
    if (j + kv <= n)
      for (int i = 1 + lane; i <= kl; i += 32) ABr(ab, ldab, i, j + kv) = 0.0;
    __syncwarp();
    const int km = min(kl, n - j);
    // ISAMAX: first index of the largest |a|
    double best = -1.0;
    int bi = 1 << 30;
    for (int i = 1 + lane; i <= km + 1; i += 32) {
      double v = fabs(ABr(ab, ldab, kv + i, j));
      if (v > best) {
        best = v;
        bi = i;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      double ob = __shfl_xor_sync(0xffffffffu, best, o);
      int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    const int jp = bi;
    if (lane == 0) ipiv[j - 1] = jp + j - 1;
    const double piv = ABr(ab, ldab, kv + jp, j);
    __syncwarp();
    if (piv != 0.0) {
      ju = max(ju, min(j + ku + jp - 1, n));
      if (jp != 1) {
        for (int cc = lane; cc < ju - j + 1; cc += 32) {
          double t1 = ABr(ab, ldab, kv + jp - cc, j + cc);
          ABr(ab, ldab, kv + jp - cc, j + cc) = ABr(ab, ldab, kv + 1 - cc, j + cc);
          ABr(ab, ldab, kv + 1 - cc, j + cc) = t1;
        }
      }
      __syncwarp();
      if (km > 0) {
        const double rcp = __ddiv_rn(1.0, ABr(ab, ldab, kv + 1, j));
        for (int i = 1 + lane; i <= km; i += 32) ABr(ab, ldab, kv + 1 + i, j) = rmul(rcp, ABr(ab, ldab, kv + 1 + i, j));
        __syncwarp();
        if (ju > j) {
          for (int jj = 1 + lane; jj <= ju - j; jj += 32) {
            double y = ABr(ab, ldab, kv + 1 - jj, j + jj);
            if (y != 0.0) {
              double temp = -y;
              for (int ii = 1; ii <= km; ++ii) {
                double& x = ABr(ab, ldab, kv + 1 + ii - jj, j + jj);
                x = radd(x, rmul(ABr(ab, ldab, kv + 1 + ii, j), temp));
              }
            }
          }
        }
        __syncwarp();
      }
    } else if (info == 0) {
      info = j;
    }
  }
  if (lane == 0) fa.info[s] = info;
}

// ===========================================================================
// Warp-cooperative banded solve (SGBTRS 'N' + STBSV, bandludcmp.f:883-1069)
// for nr right-hand sides b[r*n + row] in shared memory; same arithmetic as
// the reference (no FMA) so results equal the CPU ones bit for bit.
// ===========================================================================
__device__ void band_solve_warp(const double* __restrict__ ab, const int* __restrict__ ipiv, double* b, int nr,
                                int n, int kl, int ku, int lane) {
  // The factor entries a step needs do not depend on the data, so they are
  // fetched PF steps ahead into a register ring (indices are compile-time
  // constants after unrolling), hiding the global-memory latency that would
  // otherwise stall every step of the sequential sweep.
  constexpr int PF = 8;
  const int ldab = 2 * kl + ku + 1;
  const int kd = ku + kl + 1;
  const int i0 = lane + 1, i1 = lane + 33;
  int rl[PF];
  double rm0[PF], rm1[PF];
#pragma unroll
  for (int d = 0; d < PF; ++d) {
    const int j = 1 + d;
    rl[d] = 0;
    rm0[d] = rm1[d] = 0.0;
    if (j <= n - 1) {
      const int lm = min(kl, n - j);
      const double* col = ab + (size_t)ldab * (j - 1);
      rl[d] = __ldg(ipiv + j - 1);
      if (i0 <= lm) rm0[d] = __ldg(col + kd + i0 - 1);
      if (i1 <= lm) rm1[d] = __ldg(col + kd + i1 - 1);
    }
  }
  for (int jb = 1; jb <= n - 1; jb += PF) {
#pragma unroll
    for (int d = 0; d < PF; ++d) {
      const int j = jb + d;
      if (j <= n - 1) {
        const int lm = min(kl, n - j);
        const int l = rl[d];
        const double m0 = rm0[d], m1 = rm1[d];
        const int jn = j + PF;
        if (jn <= n - 1) {
          const int lmn = min(kl, n - jn);
          const double* coln = ab + (size_t)ldab * (jn - 1);
          rl[d] = __ldg(ipiv + jn - 1);
          rm0[d] = (i0 <= lmn) ? __ldg(coln + kd + i0 - 1) : 0.0;
          rm1[d] = (i1 <= lmn) ? __ldg(coln + kd + i1 - 1) : 0.0;
        }
        for (int r = 0; r < nr; ++r) {
          double* br = b + (size_t)r * n;
          const double bj = br[j - 1];
          const double bl = br[l - 1];
          const double y = (l != j) ? bl : bj;
          double nv0 = 0, nv1 = 0;
          if (i0 <= lm) {
            int row = j + i0;
            double old = (row == l) ? bj : br[row - 1];
            nv0 = (y != 0.0) ? radd(old, rmul(m0, -y)) : old;
          }
          if (i1 <= lm) {
            int row = j + i1;
            double old = (row == l) ? bj : br[row - 1];
            nv1 = (y != 0.0) ? radd(old, rmul(m1, -y)) : old;
          }
          __syncwarp();
          if (i0 <= lm) br[j + i0 - 1] = nv0;
          if (i1 <= lm) br[j + i1 - 1] = nv1;
          if (lane == 0) br[j - 1] = y;
          __syncwarp();
        }
      }
    }
  }
  // back substitution with the upper band (STBSV)
  const int k = kl + ku, kplus1 = k + 1;
  double rdg[PF], rv0[PF], rv1[PF], rv2[PF];
  // lane's rows below j are i = j-1-lane-32m; AB(kplus1-j+i, j) = col[k-1-lane-32m]
  const int o0 = k - 1 - lane, o1 = k - 1 - lane - 32, o2 = k - 1 - lane - 64;
#pragma unroll
  for (int d = 0; d < PF; ++d) {
    const int j = n - d;
    rdg[d] = rv0[d] = rv1[d] = rv2[d] = 0.0;
    if (j >= 1) {
      const double* col = ab + (size_t)ldab * (j - 1);
      rdg[d] = __ldg(col + kplus1 - 1);
      if (o0 >= 0) rv0[d] = __ldg(col + o0);
      if (o1 >= 0) rv1[d] = __ldg(col + o1);
      if (o2 >= 0) rv2[d] = __ldg(col + o2);
    }
  }
  for (int jb = n; jb >= 1; jb -= PF) {
#pragma unroll
    for (int d = 0; d < PF; ++d) {
      const int j = jb - d;
      if (j >= 1) {
        const double dg = rdg[d];
        const double v0 = rv0[d], v1 = rv1[d], v2 = rv2[d];
        const int jn = j - PF;
        if (jn >= 1) {
          const double* coln = ab + (size_t)ldab * (jn - 1);
          rdg[d] = __ldg(coln + kplus1 - 1);
          rv0[d] = (o0 >= 0) ? __ldg(coln + o0) : 0.0;
          rv1[d] = (o1 >= 0) ? __ldg(coln + o1) : 0.0;
          rv2[d] = (o2 >= 0) ? __ldg(coln + o2) : 0.0;
        }
        const int lo = max(1, j - k);
        const int ia = j - 1 - lane, ib = ia - 32, ic = ia - 64;
        for (int r = 0; r < nr; ++r) {
          double* br = b + (size_t)r * n;
          double xj = br[j - 1];
          if (xj != 0.0) {
            xj = __ddiv_rn(xj, dg);
            double n0 = 0, n1 = 0, n2 = 0;
            if (ia >= lo) n0 = rsub(br[ia - 1], rmul(xj, v0));
            if (ib >= lo) n1 = rsub(br[ib - 1], rmul(xj, v1));
            if (ic >= lo) n2 = rsub(br[ic - 1], rmul(xj, v2));
            __syncwarp();
            if (ia >= lo) br[ia - 1] = n0;
            if (ib >= lo) br[ib - 1] = n1;
            if (ic >= lo) br[ic - 1] = n2;
            if (lane == 0) br[j - 1] = xj;
            __syncwarp();
          }
        }
      }
    }
  }
}

// Legendre filter of solution columns (filtering.f:729-808, filter_legenpen),
// same order of operations as the reference.  One lane per subdomain column.
__device__ void legen_filter_cols(double* b, int nr, int n, int N, int ns, const double* __restrict__ wg,
                                  const double* __restrict__ alpol, const double* __restrict__ sigma, int lane) {
  const int nzm = N - 1;
  for (int t = lane; t < nr * ns; t += 32) {
    double* f = b + (size_t)(t / ns) * n + (size_t)(t % ns) * N;
    double af[kMaxN];
    for (int kk = 0; kk <= nzm; ++kk) {
      double sum = 0.0;
      for (int k1 = 0; k1 < N; ++k1) sum = radd(sum, rmul(rmul(wg[k1], f[k1]), alpol[kk * N + k1]));
      double a = (kk == nzm) ? rmul(rmul(0.5, (double)nzm), sum) : rmul((double)kk + 0.5, sum);
      af[kk] = rmul(a, sigma[kk]);
    }
    for (int k1 = 0; k1 < N; ++k1) {
      double sum = 0.0;
      for (int kk = 0; kk <= nzm; ++kk) sum = radd(sum, rmul(af[kk], alpol[kk * N + k1]));
      f[k1] = sum;
    }
  }
}

struct SolveTabs {
  const double* ab;      // ldab*nz per system
  const int* ipiv;       // nz per system
  const SysDesc* sys;
  const int* col_sys;    // per column (j*nxhp+ii): system index (-1: none)
  const double* wg;
  const double* alpol;   // N*N: alpol[k*N + k1] = P_k(z_k1)
  const double* sigma;   // N
  const double* meang;   // nz: 1 - fzgaus(z) (mean-u damping) or null
  const int* col_order;  // columns sorted by kx^2+ky^2, so neighbouring warps share a factor
};

// K_G: viscous/diffusive solves.  role 0: u and v (4 RHS, one factor),
// role 1: w, role 2: rho.  Warp per column.
template <typename T>
__global__ void k_visc(Geo g, SolveTabs tb, T* __restrict__ F0, T* __restrict__ F1, double rdiv, int role, int cpen,
                       int meanu) {
  extern __shared__ __align__(16) double sm[];
  const int warps = blockDim.x / 32;
  const int wid = threadIdx.x / 32, lane = threadIdx.x & 31;
  const int cw = blockIdx.x * warps + wid;
  const int ncol = g.nxhp * g.ny;
  if (cw >= ncol) return;
  const int c = tb.col_order[cw];
  const int n = g.nz, N = g.N;
  const int nr = role == 0 ? 4 : 2;
  double* b = sm + (size_t)wid * 4 * n;
  const int j = c / g.nxhp, ii = c % g.nxhp;
  const bool lzero = (ii == 0 && j == 0);
  const int s = tb.col_sys[c];
  T* Fs[2] = {F0, F1};
  if (s < 0) {  // w of the (0,0) mode is zero (calcuvwt.f:488-496)
    for (int k = lane; k < n; k += 32) {
      F0[fidx<T>(g, 2 * ii, j, k)] = 0;
      F0[fidx<T>(g, 2 * ii + 1, j, k)] = 0;
    }
    return;
  }
  const SysDesc sd = tb.sys[s];
  const double eps = sd.eps;
  for (int r = 0; r < nr; ++r) {
    T* F = Fs[r / 2];
    int part = r & 1;
    for (int k = lane; k < n; k += 32) {
      double x = (double)F[fidx<T>(g, 2 * ii + part, j, k)];
      double rh = -__ddiv_rn(x, rdiv);
      b[(size_t)r * n + k] = -rmul(rh, eps);
    }
  }
  __syncwarp();
  if (lane == 0) {
    // homogeneous boundary values: Dirichlet adds tau*0, Neumann tau*0*eps
    for (int r = 0; r < nr; ++r) {
      double* br = b + (size_t)r * n;
      br[0] = sd.ifbcbot == 0 ? radd(br[0], rmul(sd.tau1_bot, 0.0)) : rsub(br[0], rmul(rmul(sd.tau1_bot, 0.0), eps));
      br[n - 1] = sd.ifbctop == 0 ? radd(br[n - 1], rmul(sd.tau2_top, 0.0))
                                  : radd(br[n - 1], rmul(rmul(sd.tau2_top, 0.0), eps));
    }
  }
  __syncwarp();
  const int ldab = 3 * N + 1;
  band_solve_warp(tb.ab + (size_t)s * ldab * n, tb.ipiv + (size_t)s * n, b, nr, n, N, N, lane);
  if (cpen) {
    legen_filter_cols(b, nr, n, N, g.ns, tb.wg, tb.alpol, tb.sigma, lane);
    __syncwarp();
  }
  for (int r = 0; r < nr; ++r) {
    T* F = Fs[r / 2];
    int part = r & 1;
    for (int k = lane; k < n; k += 32) {
      double x = b[(size_t)r * n + k];
      if (role == 0 && r < 2 && lzero && meanu) x = rmul(tb.meang[k], x);
      F[fidx<T>(g, 2 * ii + part, j, k)] = (T)x;
    }
  }
}

// ===========================================================================
// Block-inverse solve of the viscous / diffusive penalty systems.
// The penalty matrix A is block diagonal in N x N subdomain blocks A_ks, plus
// coupling in the first row of block ks to all of block ks-1 (vector c_ks)
// and in its last row to all of block ks+1 (vector d_ks).  With
// y = A_ks^-1 b_ks, p_ks = A_ks^-1 e_0, q_ks = A_ks^-1 e_{N-1}:
//     x_ks = y_ks - p_ks sigma_ks - q_ks tau_ks,
//     sigma_ks = c_ks . x_{ks-1},  tau_ks = d_ks . x_{ks+1},
// and the 2(ns-1) interface scalars solve a small dense system M z = r.
// A_ks^-1 is formed once per system (FP64 Gauss-Jordan, partial pivoting),
// stored column major per block in TI (float for the mixed path).
// ===========================================================================
struct BlockInv {
  // per system: nb distinct blocks of N*N, [block][col][row].  Subdomain ks
  // uses block bmap[ks]: a block is fixed by epsilon, the subdomain height and
  // whether it has neighbours below and above, so with equal heights the
  // interior subdomains share one inverse.
  const void* ainv;
  int nb;
  int bmap[IW_MAX_SUBD];
  const double* cvec;   // per system: ns*N (c_ks, ks>=1)
  const double* dvec;   // per system: ns*N (d_ks, ks<=ns-2)
  const double* minv;   // per system: m*m, m = 2(ns-1), row major
  const double* pen;    // per system: 6*ns penalty parameters
  const SysDesc* sys;
  const int* col_sys;
  const int* col_order;
  const double* lvec;   // per system: m*N left vectors (see k_solve_cta)
};

// warp per (system, block): invert A_ks from the assembled band
__global__ void k_block_invert(Geo g, const double* __restrict__ ab, int nsys, double* __restrict__ ainv64,
                               double* __restrict__ cvec, double* __restrict__ dvec) {
  extern __shared__ __align__(16) double smi[];
  const int warps = blockDim.x / 32, wid = threadIdx.x / 32, lane = threadIdx.x & 31;
  const int task = blockIdx.x * warps + wid;
  const int N = g.N, ns = g.ns, n = g.nz, ldab = 3 * N + 1;
  if (task >= nsys * ns) return;
  const int s = task / ns, ks = task % ns, km = ks * N;
  const double* a = ab + (size_t)s * ldab * n;
  double* M = smi + (size_t)wid * N * 2 * N;  // row major N x 2N
  auto AB = [&](int r, int c) -> double {     // 0-based global (r, c)
    int br = 2 * N + r - c;                    // 0-based band row
    if (br < 0 || br >= ldab) return 0.0;
    return a[(size_t)br + (size_t)ldab * c];
  };
  for (int t = lane; t < N * 2 * N; t += 32) {
    int r = t / (2 * N), c = t % (2 * N);
    M[t] = c < N ? AB(km + r, km + c) : (c - N == r ? 1.0 : 0.0);
  }
  for (int k = lane; k < N; k += 32) {
    cvec[((size_t)s * ns + ks) * N + k] = ks > 0 ? AB(km, km - N + k) : 0.0;
    dvec[((size_t)s * ns + ks) * N + k] = ks < ns - 1 ? AB(km + N - 1, km + N + k) : 0.0;
  }
  __syncwarp();
  for (int col = 0; col < N; ++col) {
    // pivot: largest |M[r][col]|, r >= col
    double best = -1.0;
    int bi = col;
    for (int r = col + lane; r < N; r += 32) {
      double v = fabs(M[r * 2 * N + col]);
      if (v > best) {
        best = v;
        bi = r;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      double ob = __shfl_xor_sync(0xffffffffu, best, o);
      int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (bi != col)
      for (int c = lane; c < 2 * N; c += 32) {
        double t = M[col * 2 * N + c];
        M[col * 2 * N + c] = M[bi * 2 * N + c];
        M[bi * 2 * N + c] = t;
      }
    __syncwarp();
    const double inv = 1.0 / M[col * 2 * N + col];
    for (int c = lane; c < 2 * N; c += 32) M[col * 2 * N + c] *= inv;
    __syncwarp();
    for (int r = 0; r < N; ++r) {
      if (r == col) continue;
      const double f = M[r * 2 * N + col];
      if (f != 0.0)
        for (int c = lane; c < 2 * N; c += 32) M[r * 2 * N + c] -= f * M[col * 2 * N + c];
    }
    __syncwarp();
  }
  double* out = ainv64 + ((size_t)s * ns + ks) * N * N;
  for (int t = lane; t < N * N; t += 32) {
    int c = t / N, r = t % N;  // column major
    out[t] = M[r * 2 * N + N + c];
  }
}

// thread per system: interface matrix M (m = 2(ns-1)) and its inverse
__global__ void k_iface_matrix(Geo g, int nsys, const double* __restrict__ ainv64, const double* __restrict__ cvec,
                               const double* __restrict__ dvec, double* __restrict__ minv, double* __restrict__ work) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = g.N, ns = g.ns, m = 2 * (ns - 1);
  if (s >= nsys || m == 0) return;
  double* A = work + (size_t)s * 2 * m * m;  // m x 2m
  for (int t = 0; t < 2 * m * m; ++t) A[t] = 0.0;
  // unknown index: sigma_ks (ks=1..ns-1) -> ks-1 ; tau_ks (ks=0..ns-2) -> ns-1+ks
  auto inv = [&](int ks, int r, int c) { return ainv64[(((size_t)s * ns + ks) * N + c) * N + r]; };
  for (int ks = 0; ks < ns; ++ks) {
    if (ks + 1 <= ns - 1) {  // row for sigma_{ks+1}
      int row = ks;          // sigma_{ks+1} index
      const double* c = cvec + ((size_t)s * ns + ks + 1) * N;
      double cp = 0, cq = 0;
      for (int k = 0; k < N; ++k) {
        cp += c[k] * inv(ks, k, 0);
        cq += c[k] * inv(ks, k, N - 1);
      }
      A[row * 2 * m + row] += 1.0;
      if (ks >= 1) A[row * 2 * m + (ks - 1)] += cp;
      if (ks <= ns - 2) A[row * 2 * m + (ns - 1 + ks)] += cq;
    }
    if (ks - 1 >= 0) {  // row for tau_{ks-1}
      int row = ns - 1 + ks - 1;
      const double* d = dvec + ((size_t)s * ns + ks - 1) * N;
      double dp = 0, dq = 0;
      for (int k = 0; k < N; ++k) {
        dp += d[k] * inv(ks, k, 0);
        dq += d[k] * inv(ks, k, N - 1);
      }
      A[row * 2 * m + row] += 1.0;
      if (ks >= 1) A[row * 2 * m + (ks - 1)] += dp;
      if (ks <= ns - 2) A[row * 2 * m + (ns - 1 + ks)] += dq;
    }
  }
  for (int r = 0; r < m; ++r) A[r * 2 * m + m + r] = 1.0;
  for (int col = 0; col < m; ++col) {
    int bi = col;
    for (int r = col + 1; r < m; ++r)
      if (fabs(A[r * 2 * m + col]) > fabs(A[bi * 2 * m + col])) bi = r;
    if (bi != col)
      for (int c = 0; c < 2 * m; ++c) {
        double t = A[col * 2 * m + c];
        A[col * 2 * m + c] = A[bi * 2 * m + c];
        A[bi * 2 * m + c] = t;
      }
    double iv = 1.0 / A[col * 2 * m + col];
    for (int c = 0; c < 2 * m; ++c) A[col * 2 * m + c] *= iv;
    for (int r = 0; r < m; ++r)
      if (r != col) {
        double f = A[r * 2 * m + col];
        if (f != 0.0)
          for (int c = 0; c < 2 * m; ++c) A[r * 2 * m + c] -= f * A[col * 2 * m + c];
      }
  }
  for (int r = 0; r < m; ++r)
    for (int c = 0; c < m; ++c) minv[(size_t)s * m * m + r * m + c] = A[r * 2 * m + m + c];
}

// ===========================================================================
// Grouped solves: one warp per task = up to G columns that share one system
// (same kx^2+ky^2, adjacent in the sorted column order).  All right-hand
// sides of the task advance together through each elimination step, so the
// factor column is fetched once per step for all of them.
// ===========================================================================
struct Task {
  int sys;    // system index (-1: no system, e.g. pressure of the (0,0) mode)
  int first;  // index into the sorted column order
  int count;  // columns in the task (<= G)
};

// SGBTRS + STBSV arithmetic for R <= RM right-hand sides b[r*n + row]
template <int RM>
__device__ void band_solve_multi(const double* __restrict__ ab, const int* __restrict__ ipiv, double* b, int R, int n,
                                 int kl, int ku, int lane) {
  constexpr int PF = 4;
  const int ldab = 2 * kl + ku + 1, kd = ku + kl + 1;
  const int i0 = lane + 1, i1 = lane + 33;
  int rl[PF];
  double rm0[PF], rm1[PF];
#pragma unroll
  for (int d = 0; d < PF; ++d) {
    const int j = 1 + d;
    rl[d] = 0;
    rm0[d] = rm1[d] = 0.0;
    if (j <= n - 1) {
      const int lm = min(kl, n - j);
      const double* col = ab + (size_t)ldab * (j - 1);
      rl[d] = __ldg(ipiv + j - 1);
      if (i0 <= lm) rm0[d] = __ldg(col + kd + i0 - 1);
      if (i1 <= lm) rm1[d] = __ldg(col + kd + i1 - 1);
    }
  }
  for (int jb = 1; jb <= n - 1; jb += PF) {
#pragma unroll
    for (int d = 0; d < PF; ++d) {
      const int j = jb + d;
      if (j <= n - 1) {
        const int lm = min(kl, n - j);
        const int l = rl[d];
        const double m0 = rm0[d], m1 = rm1[d];
        const int jn = j + PF;
        if (jn <= n - 1) {
          const int lmn = min(kl, n - jn);
          const double* coln = ab + (size_t)ldab * (jn - 1);
          rl[d] = __ldg(ipiv + jn - 1);
          rm0[d] = (i0 <= lmn) ? __ldg(coln + kd + i0 - 1) : 0.0;
          rm1[d] = (i1 <= lmn) ? __ldg(coln + kd + i1 - 1) : 0.0;
        }
        double y[RM], nv0[RM], nv1[RM];
        const int row0 = j + i0, row1 = j + i1;
#pragma unroll
        for (int r = 0; r < RM; ++r)
          if (r < R) {
            const double* br = b + (size_t)r * n;
            const double bj = br[j - 1], bl = br[l - 1];
            y[r] = (l != j) ? bl : bj;
            if (i0 <= lm) {
              const double old = (row0 == l) ? bj : br[row0 - 1];
              nv0[r] = (y[r] != 0.0) ? radd(old, rmul(m0, -y[r])) : old;
            }
            if (i1 <= lm) {
              const double old = (row1 == l) ? bj : br[row1 - 1];
              nv1[r] = (y[r] != 0.0) ? radd(old, rmul(m1, -y[r])) : old;
            }
          }
        __syncwarp();
#pragma unroll
        for (int r = 0; r < RM; ++r)
          if (r < R) {
            double* br = b + (size_t)r * n;
            if (i0 <= lm) br[row0 - 1] = nv0[r];
            if (i1 <= lm) br[row1 - 1] = nv1[r];
            if (lane == 0) br[j - 1] = y[r];
          }
        __syncwarp();
      }
    }
  }
  const int k = kl + ku, kplus1 = k + 1;
  double rdg[PF], rv0[PF], rv1[PF], rv2[PF];
  const int o0 = k - 1 - lane, o1 = k - 1 - lane - 32, o2 = k - 1 - lane - 64;
#pragma unroll
  for (int d = 0; d < PF; ++d) {
    const int j = n - d;
    rdg[d] = rv0[d] = rv1[d] = rv2[d] = 0.0;
    if (j >= 1) {
      const double* col = ab + (size_t)ldab * (j - 1);
      rdg[d] = __ldg(col + kplus1 - 1);
      if (o0 >= 0) rv0[d] = __ldg(col + o0);
      if (o1 >= 0) rv1[d] = __ldg(col + o1);
      if (o2 >= 0) rv2[d] = __ldg(col + o2);
    }
  }
  for (int jb = n; jb >= 1; jb -= PF) {
#pragma unroll
    for (int d = 0; d < PF; ++d) {
      const int j = jb - d;
      if (j >= 1) {
        const double dg = rdg[d];
        const double v0 = rv0[d], v1 = rv1[d], v2 = rv2[d];
        const int jn = j - PF;
        if (jn >= 1) {
          const double* coln = ab + (size_t)ldab * (jn - 1);
          rdg[d] = __ldg(coln + kplus1 - 1);
          rv0[d] = (o0 >= 0) ? __ldg(coln + o0) : 0.0;
          rv1[d] = (o1 >= 0) ? __ldg(coln + o1) : 0.0;
          rv2[d] = (o2 >= 0) ? __ldg(coln + o2) : 0.0;
        }
        const int lo = max(1, j - k);
        const int ia = j - 1 - lane, ib = ia - 32, ic = ia - 64;
        double xj[RM], n0[RM], n1[RM], n2[RM];
#pragma unroll
        for (int r = 0; r < RM; ++r)
          if (r < R) {
            const double* br = b + (size_t)r * n;
            xj[r] = br[j - 1];
            if (xj[r] != 0.0) {
              xj[r] = __ddiv_rn(xj[r], dg);
              if (ia >= lo) n0[r] = rsub(br[ia - 1], rmul(xj[r], v0));
              if (ib >= lo) n1[r] = rsub(br[ib - 1], rmul(xj[r], v1));
              if (ic >= lo) n2[r] = rsub(br[ic - 1], rmul(xj[r], v2));
            }
          }
        __syncwarp();
#pragma unroll
        for (int r = 0; r < RM; ++r)
          if (r < R && xj[r] != 0.0) {
            double* br = b + (size_t)r * n;
            if (ia >= lo) br[ia - 1] = n0[r];
            if (ib >= lo) br[ib - 1] = n1[r];
            if (ic >= lo) br[ic - 1] = n2[r];
            if (lane == 0) br[j - 1] = xj[r];
          }
        __syncwarp();
      }
    }
  }
}

// K_F grouped: pressure for the columns of one task (calcuvwt.f:87-229)
template <typename T, int G>
__global__ void k_press_g(Geo g, SolveTabs tb, const Task* __restrict__ tasks, int ntask, T* __restrict__ U,
                          T* __restrict__ V, T* __restrict__ W, const double* __restrict__ wnl,
                          const double* __restrict__ wvr, int cpen, int kstart) {
  extern __shared__ __align__(16) double sm[];
  const int warps = blockDim.x / 32, wid = threadIdx.x / 32, lane = threadIdx.x & 31;
  const int t = blockIdx.x * warps + wid;
  if (t >= ntask) return;
  const Task tk = tasks[t];
  const int n = g.nz, N = g.N;
  double* B = sm + (size_t)wid * 2 * G * n;
  const int R = 2 * tk.count;
  const double dt = g.dt;
  const int s = tk.sys;
  if (s >= 0) {
    const SysDesc sd = tb.sys[s];
    const double eps = sd.eps;
    for (int ci = 0; ci < tk.count; ++ci) {
      const int c = tb.col_order[tk.first + ci];
      const int j = c / g.nxhp, ii = c % g.nxhp;
      const double xw = g.xw[ii], yw = g.yw[j];
      double* rr = B + (size_t)(2 * ci) * n;
      double* ri = rr + n;
      for (int k = lane; k < n; k += 32) {
        const int ks = k / N, k1 = k % N;
        double sr = 0.0, si = 0.0;
        for (int k2 = 0; k2 < N; ++k2) {
          const double dd = g.D[k1 * N + k2];
          sr = radd(sr, rmul(dd, (double)W[fidx<T>(g, 2 * ii, j, ks * N + k2)]));
          si = radd(si, rmul(dd, (double)W[fidx<T>(g, 2 * ii + 1, j, ks * N + k2)]));
        }
        const double fac = g.hfac[ks];
        const double dwr = rmul(sr, fac), dwi = rmul(si, fac);
        const double ur = (double)U[fidx<T>(g, 2 * ii, j, k)], ui = (double)U[fidx<T>(g, 2 * ii + 1, j, k)];
        const double vr = (double)V[fidx<T>(g, 2 * ii, j, k)], vi = (double)V[fidx<T>(g, 2 * ii + 1, j, k)];
        double dr = radd(radd(0.0, -rmul(xw, ui)), -rmul(yw, vi));
        double di = radd(radd(0.0, rmul(xw, ur)), rmul(yw, vr));
        dr = radd(dr, dwr);
        di = radd(di, dwi);
        rr[k] = -rmul(__ddiv_rn(dr, dt), eps);
        ri[k] = -rmul(__ddiv_rn(di, dt), eps);
      }
      __syncwarp();
      if (lane == 0) {
        const size_t p1 = (size_t)g.nxpp * j + 2 * ii, p2 = (size_t)g.nxpp * (j + g.ny) + 2 * ii;
        const double bcrbot = radd(wnl[p1], wvr[p1]), bcibot = radd(wnl[p1 + 1], wvr[p1 + 1]);
        const double bcrtop = radd(wnl[p2], wvr[p2]), bcitop = radd(wnl[p2 + 1], wvr[p2 + 1]);
        rr[0] = rsub(rr[0], rmul(rmul(sd.tau1_bot, bcrbot), eps));
        ri[0] = rsub(ri[0], rmul(rmul(sd.tau1_bot, bcibot), eps));
        rr[n - 1] = radd(rr[n - 1], rmul(rmul(sd.tau2_top, bcrtop), eps));
        ri[n - 1] = radd(ri[n - 1], rmul(rmul(sd.tau2_top, bcitop), eps));
      }
      __syncwarp();
    }
    const int ldab = 3 * N + 1;
    band_solve_multi<2 * G>(tb.ab + (size_t)s * ldab * n, tb.ipiv + (size_t)s * n, B, R, n, N, N, lane);
    if (cpen) {
      legen_filter_cols(B, R, n, N, g.ns, tb.wg, tb.alpol, tb.sigma, lane);
      __syncwarp();
    }
  } else {
    for (int q = lane; q < R * n; q += 32) B[q] = 0.0;
    __syncwarp();
  }
  for (int ci = 0; ci < tk.count; ++ci) {
    const int c = tb.col_order[tk.first + ci];
    const int j = c / g.nxhp, ii = c % g.nxhp;
    const bool lzero = (ii == 0 && j == 0);
    const double dtx = rmul(dt, g.xw[ii]), dty = rmul(dt, g.yw[j]);
    const double* rr = B + (size_t)(2 * ci) * n;
    const double* ri = rr + n;
    for (int k = lane; k < n; k += 32) {
      const size_t pr = fidx<T>(g, 2 * ii, j, k), pi = pr + 1;
      if (k < kstart) {
        U[pr] = 0;
        U[pi] = 0;
        V[pr] = 0;
        V[pi] = 0;
        W[pr] = 0;
        W[pi] = 0;
        continue;
      }
      const double phr = rr[k], phi = ri[k];
      const double ur = (double)U[pr], ui = (double)U[pi], vr = (double)V[pr], vi = (double)V[pi];
      double wbr = 0, wbi = 0;
      if (!lzero) {
        const int ks = k / N, k1 = k % N;
        double sr = 0.0, si = 0.0;
        for (int k2 = 0; k2 < N; ++k2) {
          const double dd = g.D[k1 * N + k2];
          sr = radd(sr, rmul(dd, rr[ks * N + k2]));
          si = radd(si, rmul(dd, ri[ks * N + k2]));
        }
        const double fac = g.hfac[ks];
        wbr = rsub((double)W[pr], rmul(dt, rmul(sr, fac)));
        wbi = rsub((double)W[pi], rmul(dt, rmul(si, fac)));
      }
      U[pr] = (T)rsub(ur, rsub(rmul(0.0, phr), rmul(dtx, phi)));
      U[pi] = (T)rsub(ui, radd(rmul(0.0, phi), rmul(dtx, phr)));
      V[pr] = (T)rsub(vr, rsub(rmul(0.0, phr), rmul(dty, phi)));
      V[pi] = (T)rsub(vi, radd(rmul(0.0, phi), rmul(dty, phr)));
      W[pr] = (T)wbr;
      W[pi] = (T)wbi;
    }
  }
}

// ===========================================================================
// Block-inverse solve, one CTA per task (row parallel).
//
// A = blockdiag(A_0..A_{ns-1}) + interface couplings (first row of block ks
// couples to the last row of ks-1 through c_ks, last row of ks to the first
// row of ks+1 through d_ks).  With y = blockdiag^-1 b the interface unknowns
// solve M z = r, r_e = <c_{e+1}, y_e> (e < ns-1), <d_t, y_{t+1}> (e = ns-1+t),
// and x = y - A_ks^-1 e_0 z_{ks-1} - A_ks^-1 e_{N-1} z_{ns-1+ks}.
// Because <c, A^-1 b> = <A^-T c, b>, the left vectors lvec = A^-T c, A^-T d
// are precomputed per system, so r comes straight from b and x from one sweep
// in which every inverse entry is read once (coalesced) and used for all R
// right-hand sides.  Each thread owns whole rows.
// ===========================================================================
constexpr int kSolveThreads = 128;

// (re, im) pair of one complex value stored as two T
template <typename T>
struct Pair;
template <>
struct Pair<float> {
  typedef float2 t;
};
template <>
struct Pair<double> {
  typedef double2 t;
};


// dst = (accum ? dst : 0) + A^-1 src for R right-hand sides of length n.
// rz, zz: R*m doubles of shared scratch.  Ends synchronised.
template <int R>
__device__ void bi_apply_cta(const Geo& g, const double* __restrict__ ainv, const int* bmap,
                             const double* __restrict__ lvec, const double* __restrict__ minv, const double* src,
                             double* dst, double* rz, double* zz, bool accum) {
  const int N = g.N, ns = g.ns, n = g.nz, m = 2 * (ns - 1);
  const int tid = threadIdx.x;
  if (m > 0) {
    for (int q = tid; q < m * R; q += kSolveThreads) {
      const int r = q / m, e = q - r * m;
      const int blk = e < ns - 1 ? e : e - (ns - 1) + 1;
      const double* lv = lvec + (size_t)e * N;
      const double* sv = src + (size_t)r * n + blk * N;
      double acc = 0.0;
#pragma unroll 4
      for (int k = 0; k < N; ++k) acc += lv[k] * sv[k];
      rz[q] = acc;
    }
    __syncthreads();
    for (int q = tid; q < m * R; q += kSolveThreads) {
      const int r = q / m, e = q - r * m;
      const double* mr = minv + (size_t)e * m;
      const double* rr = rz + r * m;
      double z = 0.0;
#pragma unroll 4
      for (int c = 0; c < m; ++c) z += mr[c] * rr[c];
      zz[q] = z;
    }
    __syncthreads();
  }
  for (int row = tid; row < n; row += kSolveThreads) {
    const int ks = row / N, kk = row - ks * N;
    const double* ai = ainv + (size_t)bmap[ks] * N * N + kk;
    const double* sv = src + ks * N;
    double acc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = 0.0;
#pragma unroll 8
    for (int c = 0; c < N; ++c) {
      const double a = __ldg(ai + (size_t)c * N);
#pragma unroll
      for (int r = 0; r < R; ++r) acc[r] += a * sv[(size_t)r * n + c];
    }
    const double p = ks >= 1 ? __ldg(ai) : 0.0;
    const double q = ks <= ns - 2 ? __ldg(ai + (size_t)(N - 1) * N) : 0.0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      double x = acc[r];
      if (ks >= 1) x -= p * zz[r * m + ks - 1];
      if (ks <= ns - 2) x -= q * zz[r * m + ns - 1 + ks];
      double* d = dst + (size_t)r * n + row;
      *d = accum ? *d + x : x;
    }
  }
  __syncthreads();
}

// b -= A x for R right-hand sides (matrix free, FP64).  D2t/Dt: transposed
// differentiation matrices (Dt[k*N + k1] = D[k1][k]).
template <int R>
__device__ void sub_A_cta(const Geo& g, const double* __restrict__ D2t, const double* __restrict__ zh, double eps,
                          const double* __restrict__ pen, const double* x, double* b) {
  const int N = g.N, ns = g.ns, n = g.nz;
  for (int row = threadIdx.x; row < n; row += kSolveThreads) {
    const int ks = row / N, k1 = row - ks * N, km = ks * N;
    const double h2 = 2.0 / zh[ks];
    double s2[R];
#pragma unroll
    for (int r = 0; r < R; ++r) s2[r] = 0.0;
#pragma unroll 8
    for (int k = 0; k < N; ++k) {
      const double d = __ldg(D2t + k * N + k1);
#pragma unroll
      for (int r = 0; r < R; ++r) s2[r] += d * x[(size_t)r * n + km + k];
    }
    const double ee = eps * (h2 * h2);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const double* xr = x + (size_t)r * n;
      double v = xr[row] - ee * s2[r];
      if (k1 == 0) {
        const double pa = pen[ks], pb = pen[ns + ks], t1 = pen[4 * ns + ks];
        double s0 = 0;
        for (int k = 0; k < N; ++k) s0 += g.D[k] * xr[km + k];
        v += t1 * pa * xr[km] - t1 * pb * eps * h2 * s0;
        if (ks > 0) {
          const double hl = 2.0 / zh[ks - 1];
          double sl = 0;
          for (int k = 0; k < N; ++k) sl += g.D[(N - 1) * N + k] * xr[km - N + k];
          v += -0.5 * t1 * pa * xr[km] + 0.5 * t1 * pb * eps * h2 * s0 - 0.5 * t1 * pa * xr[km - 1] +
               0.5 * t1 * pb * eps * hl * sl;
        }
      }
      if (k1 == N - 1) {
        const double pg = pen[2 * ns + ks], pd = pen[3 * ns + ks], t2 = pen[5 * ns + ks];
        double s1 = 0;
        for (int k = 0; k < N; ++k) s1 += g.D[(N - 1) * N + k] * xr[km + k];
        v += t2 * pg * xr[km + N - 1] + t2 * pd * eps * h2 * s1;
        if (ks < ns - 1) {
          const double hr = 2.0 / zh[ks + 1];
          double sr = 0;
          for (int k = 0; k < N; ++k) sr += g.D[k] * xr[km + N + k];
          v += -0.5 * t2 * pg * xr[km + N - 1] - 0.5 * t2 * pd * eps * h2 * s1 - 0.5 * t2 * pg * xr[km + N] -
               0.5 * t2 * pd * eps * hr * sr;
        }
      }
      b[(size_t)r * n + row] -= v;
    }
  }
  __syncthreads();
}

// dst[r][row] = sum_j L[kk][j] src[r][ks*N + j]: the Legendre filter of every
// subdomain (filtering.f:1225-1243 with the precombined matrix; Lt = L^T).
template <int R>
__device__ void legen_filter_cta(const Geo& g, const double* __restrict__ Lt, const double* src, double* dst) {
  const int N = g.N, n = g.nz;
  for (int row = threadIdx.x; row < n; row += kSolveThreads) {
    const int ks = row / N, kk = row - ks * N;
    const double* sv = src + ks * N;
    double acc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = 0.0;
#pragma unroll 8
    for (int j = 0; j < N; ++j) {
      const double l = __ldg(Lt + j * N + kk);
#pragma unroll
      for (int r = 0; r < R; ++r) acc[r] += l * sv[(size_t)r * n + j];
    }
#pragma unroll
    for (int r = 0; r < R; ++r) dst[(size_t)r * n + row] = acc[r];
  }
  __syncthreads();
}

// Solve of one task: <= R/per columns sharing system tk.sys, per = 4 right-hand
// sides per column for role 0 (u, v re/im), 2 otherwise; unused ones are zero.
// role 0: u/v (F0, F1), 1: w (F0), 2: rho (F0), 3: pressure from u*,v*,w*
// (F0, F1, F2) followed by the projection (calcuvwt.f:87-229, 826-901).
// refine: one FP64 residual sweep x += A^-1 (b - A x).
template <typename T, int R>
__global__ void __launch_bounds__(kSolveThreads) k_solve_cta(
    Geo g, BlockInv bi, SolveTabs tb, const Task* __restrict__ tasks, T* __restrict__ F0, T* __restrict__ F1,
    T* __restrict__ F2, double rdiv, int role, int cpen, int meanu, int refine, const double* __restrict__ Dt,
    const double* __restrict__ D2t, const double* __restrict__ Lt, const double* __restrict__ zh,
    const double* __restrict__ wnl, const double* __restrict__ wvr, int kstart) {
  extern __shared__ __align__(16) double sm[];
  __shared__ int cj[R], cii[R];
  const Task tk = tasks[blockIdx.x];
  const int n = g.nz, N = g.N, ns = g.ns, m = 2 * (ns - 1);
  const int tid = threadIdx.x;
  double* b = sm;
  double* x = b + (size_t)R * n;
  double* rz = x + (size_t)R * n;
  double* zz = rz + (size_t)R * (m > 0 ? m : 1);
  // role 3: u*, v*, w* of the task's columns, [field][r][k], read from global
  // memory once for both the divergence and the projection
  T* fv = (T*)(zz + (size_t)R * (m > 0 ? m : 1));
  const int per = role == 0 ? 4 : 2;
  const int ncols = R / per;  // column slots per task
  const int s = tk.sys;
  const int ncolt = tk.count;
  const double dt = g.dt;
  if (tid < ncols) {
    const int c = tid < ncolt ? tb.col_order[tk.first + tid] : -1;
    cj[tid] = c < 0 ? -1 : c / g.nxhp;
    cii[tid] = c < 0 ? -1 : c % g.nxhp;
  }
  __syncthreads();
  if (role == 3) {
    // one 8-byte (re, im) load per field and column, all in flight at once
    typedef typename Pair<T>::t P2;
    for (int k = tid; k < n; k += kSolveThreads) {
#pragma unroll
      for (int ci = 0; ci < R / 2; ++ci) {
        P2 u2 = {0, 0}, v2 = {0, 0}, w2 = {0, 0};
        if (cj[ci] >= 0) {
          const size_t p = fidx<T>(g, 2 * cii[ci], cj[ci], k);
          u2 = *(const P2*)(F0 + p);
          v2 = *(const P2*)(F1 + p);
          w2 = *(const P2*)(F2 + p);
        }
        fv[(size_t)(2 * ci) * n + k] = u2.x;
        fv[(size_t)(2 * ci + 1) * n + k] = u2.y;
        fv[(size_t)(R + 2 * ci) * n + k] = v2.x;
        fv[(size_t)(R + 2 * ci + 1) * n + k] = v2.y;
        fv[(size_t)(2 * R + 2 * ci) * n + k] = w2.x;
        fv[(size_t)(2 * R + 2 * ci + 1) * n + k] = w2.y;
      }
    }
    __syncthreads();
  }
  if (s < 0 && role != 3) {  // w of the (0,0) mode is zero
    for (int ci = 0; ci < ncolt; ++ci)
      for (int k = tid; k < n; k += kSolveThreads) {
        F0[fidx<T>(g, 2 * cii[ci], cj[ci], k)] = 0;
        F0[fidx<T>(g, 2 * cii[ci] + 1, cj[ci], k)] = 0;
      }
    return;
  }
  const double* res = x;
  if (s < 0) {  // pressure of the (0,0) mode: phi = 0
    for (int q = tid; q < R * n; q += kSolveThreads) x[q] = 0.0;
    __syncthreads();
  } else {
    const SysDesc sd = bi.sys[s];
    const double eps = sd.eps;
    if (role == 3) {
      for (int k = tid; k < n; k += kSolveThreads) {  // w* columns into x (scratch)
#pragma unroll
        for (int r = 0; r < R; ++r) x[(size_t)r * n + k] = (double)fv[(size_t)(2 * R + r) * n + k];
      }
      __syncthreads();
      for (int k = tid; k < n; k += kSolveThreads) {
        const int ks = k / N, k1 = k - ks * N;
        double dw[R];
#pragma unroll
        for (int r = 0; r < R; ++r) dw[r] = 0.0;
        for (int k2 = 0; k2 < N; ++k2) {
          const double dd = __ldg(Dt + k2 * N + k1);
#pragma unroll
          for (int r = 0; r < R; ++r) dw[r] += dd * x[(size_t)r * n + ks * N + k2];
        }
        const double fac = g.hfac[ks];
#pragma unroll
        for (int ci = 0; ci < R / 2; ++ci) {
          double vr = 0.0, vi = 0.0;
          if (cj[ci] >= 0) {
            const int j = cj[ci], ii = cii[ci];
            const double ur = (double)fv[(size_t)(2 * ci) * n + k], ui = (double)fv[(size_t)(2 * ci + 1) * n + k];
            const double wr = (double)fv[(size_t)(R + 2 * ci) * n + k];
            const double wi = (double)fv[(size_t)(R + 2 * ci + 1) * n + k];
            const double xw = g.xw[ii], yw = g.yw[j];
            const double dr = -(xw * ui) - (yw * wi) + dw[2 * ci] * fac;
            const double di = (xw * ur) + (yw * wr) + dw[2 * ci + 1] * fac;
            vr = -((dr / dt) * eps);
            vi = -((di / dt) * eps);
            if (k == 0) {
              const size_t p1 = (size_t)g.nxpp * j + 2 * ii;
              vr -= (sd.tau1_bot * (wnl[p1] + wvr[p1])) * eps;
              vi -= (sd.tau1_bot * (wnl[p1 + 1] + wvr[p1 + 1])) * eps;
            }
            if (k == n - 1) {
              const size_t p2 = (size_t)g.nxpp * (j + g.ny) + 2 * ii;
              vr += (sd.tau2_top * (wnl[p2] + wvr[p2])) * eps;
              vi += (sd.tau2_top * (wnl[p2 + 1] + wvr[p2 + 1])) * eps;
            }
          }
          b[(size_t)(2 * ci) * n + k] = vr;
          b[(size_t)(2 * ci + 1) * n + k] = vi;
        }
      }
    } else {
      for (int k = tid; k < n; k += kSolveThreads) {
        double v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int ci = r / per, rr = r - ci * per;
          const T* F = (role == 0 && rr >= 2) ? F1 : F0;
          v[r] = cj[ci] >= 0 ? (double)F[fidx<T>(g, 2 * cii[ci] + (rr & 1), cj[ci], k)] : 0.0;
        }
#pragma unroll
        for (int r = 0; r < R; ++r) b[(size_t)r * n + k] = -(-(v[r] / rdiv) * eps);
      }
    }
    __syncthreads();
    const double* ainv = (const double*)bi.ainv + (size_t)s * bi.nb * N * N;
    const double* lv = bi.lvec + (size_t)s * (m > 0 ? m : 1) * N;
    const double* mi = bi.minv + (size_t)s * (m > 0 ? m * m : 1);
    bi_apply_cta<R>(g, ainv, bi.bmap, lv, mi, b, x, rz, zz, false);
    if (refine) {
      sub_A_cta<R>(g, D2t, zh, eps, bi.pen + (size_t)s * 6 * ns, x, b);
      bi_apply_cta<R>(g, ainv, bi.bmap, lv, mi, b, x, rz, zz, true);
    }
    if (cpen) {
      legen_filter_cta<R>(g, Lt, x, b);
      res = b;
    }
  }
  // write back
  if (role == 3) {
    for (int k = tid; k < n; k += kSolveThreads) {
      const int ks = k / N, k1 = k - ks * N;
      double dz[R];
#pragma unroll
      for (int r = 0; r < R; ++r) dz[r] = 0.0;
      for (int k2 = 0; k2 < N; ++k2) {
        const double dd = __ldg(Dt + k2 * N + k1);
#pragma unroll
        for (int r = 0; r < R; ++r) dz[r] += dd * res[(size_t)r * n + ks * N + k2];
      }
      const double fac = g.hfac[ks];
#pragma unroll
      for (int ci = 0; ci < R / 2; ++ci) {
        if (cj[ci] < 0) continue;
        const int j = cj[ci], ii = cii[ci];
        const size_t pr = fidx<T>(g, 2 * ii, j, k), pi = pr + 1;
        if (k < kstart) {
          F0[pr] = 0;
          F0[pi] = 0;
          F1[pr] = 0;
          F1[pi] = 0;
          F2[pr] = 0;
          F2[pi] = 0;
          continue;
        }
        const double phr = res[(size_t)(2 * ci) * n + k], phi = res[(size_t)(2 * ci + 1) * n + k];
        double wbr = 0, wbi = 0;
        if (!(ii == 0 && j == 0)) {
          wbr = (double)fv[(size_t)(2 * R + 2 * ci) * n + k] - dt * (dz[2 * ci] * fac);
          wbi = (double)fv[(size_t)(2 * R + 2 * ci + 1) * n + k] - dt * (dz[2 * ci + 1] * fac);
        }
        const double dtx = dt * g.xw[ii], dty = dt * g.yw[j];
        const double ur = (double)fv[(size_t)(2 * ci) * n + k], ui = (double)fv[(size_t)(2 * ci + 1) * n + k];
        const double vr = (double)fv[(size_t)(R + 2 * ci) * n + k], vi = (double)fv[(size_t)(R + 2 * ci + 1) * n + k];
        F0[pr] = (T)(ur + dtx * phi);
        F0[pi] = (T)(ui - dtx * phr);
        F1[pr] = (T)(vr + dty * phi);
        F1[pi] = (T)(vi - dty * phr);
        F2[pr] = (T)wbr;
        F2[pi] = (T)wbi;
      }
    }
  } else {
    for (int k = tid; k < n; k += kSolveThreads) {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int ci = r / per, rr = r - ci * per;
        if (cj[ci] < 0) continue;
        T* F = (role == 0 && rr >= 2) ? F1 : F0;
        double v = res[(size_t)r * n + k];
        if (role == 0 && rr < 2 && meanu && cii[ci] == 0 && cj[ci] == 0) v = tb.meang[k] * v;
        F[fidx<T>(g, 2 * cii[ci] + (rr & 1), cj[ci], k)] = (T)v;
      }
    }
  }
}

// ===========================================================================
// System-grouped solve.  One CTA per group of columns that share one system:
// up to 4 u/v columns (16 right-hand sides) or 8 columns of w, rho or the
// pressure (16 right-hand sides).  The system's distinct inverse blocks, its
// left vectors and its interface matrix come into shared memory once per CTA
// by bulk asynchronous copies (cp.async.bulk, completion counted on an
// mbarrier) while the CTA gathers its columns, so every product reads both
// operands from shared memory.  Thread t owns row t for all 16 right-hand
// sides: one shared load of an inverse entry serves 16 multiply-adds, and the
// right-hand sides are stored [row][16], so the 16 values of one row come as
// eight 16-byte broadcasts.  The arithmetic (order of every sum, the RHS and
// projection formulas) is the one of k_solve_cta, so both give the same bits.
// Used for n <= 512 rows, filter folded into the inverses (or no filter),
// no residual sweep and a system present; k_solve_cta takes the rest.
// ===========================================================================
constexpr int kSysR = 16;
// row stride of the right-hand sides in shared memory: 16 values + 2 of padding,
// so that the 16-byte stores of consecutive rows fall on different banks
constexpr int kSysRS = kSysR + 2;
constexpr int kSysMaxRows = 512;

struct SysSmem {  // offsets (doubles) of the shared-memory regions of k_solve_sys
  size_t a, l, m, b, rz, zz, d, total;
};
__host__ __device__ inline SysSmem sys_smem(int n, int N, int ns, int nb, bool dmat, int rs = kSysRS, int ap = 0) {
  SysSmem o;
  const size_t m = 2 * (size_t)(ns - 1), m1 = m > 0 ? m : 1;
  if (ap <= 0) ap = N;
  o.a = 0;
  o.l = ((size_t)nb * N * ap + 3) & ~(size_t)1;  // room for a copy that starts one double early
  o.m = o.l + m * N;
  o.b = o.m + m * m;
  o.rz = o.b + (size_t)n * rs;
  o.zz = o.rz + kSysR * m1;
  o.d = o.zz + kSysR * m1;
  o.total = o.d + (dmat ? (((size_t)N * ap + 1) & ~(size_t)1) : 0);
  return o;
}

// 8-byte shared load.  The 16 right-hand-side values of a row are the same
// for every lane of a warp that works in one block (a broadcast): as 8-byte
// loads each costs one shared-memory wavefront, as 16-byte loads four.
__device__ __forceinline__ double lds64(const double* p) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(smem_u32(p)));
  return v;
}

// acc[r] = sum_c col[c*N] * b[(base + c)*RS + r]: one row of a block product;
// the loads go out in groups of BL
template <int BL = 8>
__device__ __forceinline__ void row_product16(const double* col, const double* bb, int N, double* acc) {
#pragma unroll
  for (int r = 0; r < kSysR; ++r) acc[r] = 0.0;
#pragma unroll 2
  for (int c = 0; c < N; ++c) {
    const double a = col[(size_t)c * N];
    const double* br = bb + (size_t)c * kSysRS;
#pragma unroll
    for (int h = 0; h < kSysR; h += BL) {
      double v[BL];
#pragma unroll
      for (int r = 0; r < BL; ++r) v[r] = lds64(br + h + r);
#pragma unroll
      for (int r = 0; r < BL; ++r) acc[h + r] += a * v[r];
    }
  }
}

// FP64 tensor-core variant of the block products (mma.sync m8n8k4, the FP64
// matrix instruction of sm_100a; tcgen05 has no FP64 kind).  A warp owns whole
// subdomains: X_ks[:, 8 nt .. 8 nt + 7] = Op_ks B_ks[:, 8 nt ..] in row tiles
// of 8, 4 columns of Op per instruction, the padding of the ragged N read as
// zeros.  Lane (g, t4) = (lane / 4, lane % 4) ends with
// X[8 mt + g][8 nt + 2 t4 + {0, 1}]: one complex value of one column.  The
// right-hand-side rows keep the stride of 18 doubles (a B fragment then takes
// four shared-memory wavefronts instead of two, but a stride of 20 would cost
// the second resident CTA per SM at C3's sizes); the operators get rows of
// tc_ap(N) doubles, which makes the five A fragments per step conflict-free.
constexpr int kTcRS = 18;
constexpr int kTcMT = 5;  // row tiles per subdomain: N <= 40

// Row stride of the operators staged for the tensor-core products: = 4
// (mod 8) doubles, so that an A fragment (8 rows x 4 columns of 8 bytes) falls
// in two shared-memory wavefronts.
__host__ __device__ inline int tc_ap(int N) {
  int a = N;
  while (a % 8 != 4) ++a;
  return a;
}

__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// acc[mt] = (Op B)[8 mt + g][8 nt + 2 t4 + {0, 1}] for Op(r, c) = op[c ap + r] and
// B(c, :) = bb[c kTcRS + :], c < N
__device__ __forceinline__ void tc_block_product(const double* op, int ap, const double* bb, int N, int nt, int lane,
                                                 double (&acc)[kTcMT][2]) {
  const int g = lane >> 2, t4 = lane & 3;
  const int MT = (N + 7) >> 3, KT = (N + 3) >> 2;
  __syncwarp();  // mma.sync wants the whole warp converged
#pragma unroll
  for (int mt = 0; mt < kTcMT; ++mt) acc[mt][0] = acc[mt][1] = 0.0;
#pragma unroll 3
  for (int kt = 0; kt < KT; ++kt) {
    const int c = kt * 4 + t4;
    const bool cin = c < N;
    const int cc = cin ? c : N - 1;  // in-range address for the padding
    const double b = cin ? bb[(size_t)cc * kTcRS + nt * 8 + g] : 0.0;
#pragma unroll
    for (int mt = 0; mt < kTcMT; ++mt) {
      if (mt < MT) {
        const int r = mt * 8 + g;
        const bool rin = r < N;
        const double a = (cin && rin) ? op[(size_t)cc * ap + (rin ? r : N - 1)] : 0.0;
        dmma884(acc[mt][0], acc[mt][1], a, b);
      }
    }
  }
}
// both halves of the 16 right-hand sides at once (each A fragment loaded once)
__device__ __forceinline__ void tc_block_product2(const double* op, int ap, const double* bb, int N, int lane,
                                                  double (&acc)[2][kTcMT][2]) {
  const int g = lane >> 2, t4 = lane & 3;
  const int MT = (N + 7) >> 3, KT = (N + 3) >> 2;
  __syncwarp();
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int mt = 0; mt < kTcMT; ++mt) acc[h][mt][0] = acc[h][mt][1] = 0.0;
#pragma unroll 3
  for (int kt = 0; kt < KT; ++kt) {
    const int c = kt * 4 + t4;
    const bool cin = c < N;
    const int cc = cin ? c : N - 1;
    const double b0 = cin ? bb[(size_t)cc * kTcRS + g] : 0.0;
    const double b1 = cin ? bb[(size_t)cc * kTcRS + 8 + g] : 0.0;
#pragma unroll
    for (int mt = 0; mt < kTcMT; ++mt) {
      if (mt < MT) {
        const int r = mt * 8 + g;
        const bool rin = r < N;
        const double a = (cin && rin) ? op[(size_t)cc * ap + (rin ? r : N - 1)] : 0.0;
        dmma884(acc[0][mt][0], acc[0][mt][1], a, b0);
        dmma884(acc[1][mt][0], acc[1][mt][1], a, b1);
      }
    }
  }
}

// role 0: u/v (4 RHS per column), 1: w, 2: rho, 3: pressure + projection.
// TC: block products on the FP64 tensor cores (N <= 40), else one row per
// thread on the FP64 pipes.
template <typename T, int ROLE, bool TC = false>
__global__ void __maxnreg__(72) k_solve_sys(
    Geo g, BlockInv bi, const Task* __restrict__ tasks, const int* __restrict__ col_order, T* __restrict__ F0,
    T* __restrict__ F1, T* __restrict__ F2, double rdiv, int meanu, const double* __restrict__ meang,
    const double* __restrict__ Dt, const double* __restrict__ wnl, const double* __restrict__ wvr, int kstart,
    int* __restrict__ err) {
  typedef typename Pair<T>::t P2;
  constexpr int R = kSysR;
  constexpr int PER = ROLE == 0 ? 4 : 2;  // right-hand sides per column
  constexpr int NC = R / PER;             // column slots
  constexpr int RS = TC ? kTcRS : kSysRS;  // right-hand-side row stride
  extern __shared__ __align__(16) double sm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int cj[NC], cii[NC];
  const Task tk = tasks[blockIdx.x];
  const int n = g.nz, N = g.N, ns = g.ns, m = 2 * (ns - 1), nb = bi.nb;
  const int tid = threadIdx.x;
  const int s = tk.sys;
  const int AP = TC ? tc_ap(N) : N;  // operator row stride in shared memory
  const SysSmem L = sys_smem(n, N, ns, nb, ROLE == 3, RS, AP);
  double* sA = sm + L.a;
  double* sL = sm + L.l;
  double* sM = sm + L.m;
  double* sb = sm + L.b;
  double* srz = sm + L.rz;
  double* szz = sm + L.zz;
  double* sD = sm + L.d;
  // the system's tables: one bulk copy each, all counted on one mbarrier
  const uintptr_t ga = (uintptr_t)((const double*)bi.ainv + (size_t)s * nb * N * N);
  const int offA = (int)((ga & 15u) >> 3);  // the copy starts one double early when ga is not 16-byte aligned
  const uint32_t bytesA = (uint32_t)((((size_t)nb * N * N + offA) * 8 + 15) & ~(size_t)15);
  const uint32_t bytesL = (uint32_t)((size_t)m * N * 8), bytesM = (uint32_t)((size_t)m * m * 8);
  if (tid == 0) mbar_init(&bar, 1);
  if (tid < NC) {
    const int c = tid < tk.count ? col_order[tk.first + tid] : -1;
    cj[tid] = c < 0 ? -1 : c / g.nxhp;
    cii[tid] = c < 0 ? -1 : c % g.nxhp;
  }
  __syncthreads();
  if (tid == 0) {
    // (the tensor-core variant stages the inverse blocks itself, below, in
    // rows of AP doubles)
    mbar_expect_tx(&bar, (TC ? 0u : bytesA) + bytesL + bytesM);
    if (!TC) bulk_g2s(sA, (const void*)(ga - (uintptr_t)offA * 8), bytesA, &bar);
    if (m > 0) {
      bulk_g2s(sL, bi.lvec + (size_t)s * m * N, bytesL, &bar);
      bulk_g2s(sM, bi.minv + (size_t)s * m * m, bytesM, &bar);
    }
  }
  if (TC) {
    const double* ag = (const double*)bi.ainv + (size_t)s * nb * N * N;
    for (int q = tid; q < nb * N * N; q += blockDim.x) {
      const int c = q / N, r = q - c * N;  // c runs over the blocks' columns
      sA[(size_t)c * AP + r] = ag[q];
    }
  }
  if (ROLE == 3) {
    if (TC) {
      for (int q = tid; q < N * N; q += blockDim.x) {
        const int c = q / N, r = q - c * N;
        sD[(size_t)c * AP + r] = Dt[q];
      }
    } else {
      for (int q = tid; q < N * N; q += blockDim.x) sD[q] = Dt[q];
    }
  }
  const double eps = bi.sys[s].eps;
  const double dt = g.dt;
  const int k = tid;
  const bool live = k < n;
  const int ks = live ? k / N : 0, kk = k - ks * N;
  // gather this row of every column: [row][16]
  if (live) {
    double v[R];
#pragma unroll
    for (int ci = 0; ci < NC; ++ci) {
      P2 a = {0, 0}, b = {0, 0};
      if (cj[ci] >= 0) {
        const size_t p = fidx<T>(g, 2 * cii[ci], cj[ci], k);
        if (ROLE == 3) {
          a = *(const P2*)(F2 + p);
        } else {
          a = *(const P2*)(F0 + p);
          if (ROLE == 0) b = *(const P2*)(F1 + p);
        }
      }
      v[PER * ci] = (double)a.x;
      v[PER * ci + 1] = (double)a.y;
      if (ROLE == 0) {
        v[PER * ci + 2] = (double)b.x;
        v[PER * ci + 3] = (double)b.y;
      }
    }
    if (ROLE != 3) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = -(-(v[r] / rdiv) * eps);
    }
    double2* d2 = (double2*)(sb + (size_t)k * RS);
#pragma unroll
    for (int q = 0; q < R / 2; ++q) d2[q] = make_double2(v[2 * q], v[2 * q + 1]);
  }
  const bool ok = mbar_wait(&bar, 0, 2000000000ull);
  if (__syncthreads_or(!ok)) {  // the tables never arrived: report, let the copies finish, leave
    if (tid == 0) err[1] = 1;
    mbar_wait(&bar, 0, 2000000000ull);
    return;
  }
  const int lane = tid & 31, wid = tid >> 5, nwarp = blockDim.x >> 5;
  if constexpr (TC) {
    if (ROLE == 3) {
      // divergence of u* per subdomain on the tensor cores, the RHS written
      // over w* in place (a warp reads and writes only its own subdomains)
      const int gq = lane >> 2, t4 = lane & 3, MT = (N + 7) >> 3;
      const SysDesc sd = bi.sys[s];
      for (int ks2 = wid; ks2 < ns; ks2 += nwarp) {
        double* bb = sb + (size_t)ks2 * N * RS;
        const double fac = g.hfac[ks2];
        for (int nt = 0; nt < 2; ++nt) {
          double tacc[kTcMT][2];
          tc_block_product(sD, AP, bb, N, nt, lane, tacc);
          __syncwarp();
          const int c0 = nt * 8 + 2 * t4, ci = c0 >> 1;
#pragma unroll
          for (int mt = 0; mt < kTcMT; ++mt) {
            const int r = mt * 8 + gq;
            if (mt >= MT || r >= N) continue;
            const int kq = ks2 * N + r;
            double vr = 0.0, vi = 0.0;
            if (cj[ci] >= 0) {
              const int j = cj[ci], ii = cii[ci];
              const size_t pr = fidx<T>(g, 2 * ii, j, kq);
              const P2 u2 = *(const P2*)(F0 + pr), w2 = *(const P2*)(F1 + pr);
              const double ur = (double)u2.x, ui = (double)u2.y;
              const double wr = (double)w2.x, wi = (double)w2.y;
              const double xw = g.xw[ii], yw = g.yw[j];
              const double dr = -(xw * ui) - (yw * wi) + tacc[mt][0] * fac;
              const double di = (xw * ur) + (yw * wr) + tacc[mt][1] * fac;
              vr = -((dr / dt) * eps);
              vi = -((di / dt) * eps);
              if (kq == 0) {
                const size_t p1 = (size_t)g.nxpp * j + 2 * ii;
                vr -= (sd.tau1_bot * (wnl[p1] + wvr[p1])) * eps;
                vi -= (sd.tau1_bot * (wnl[p1 + 1] + wvr[p1 + 1])) * eps;
              }
              if (kq == n - 1) {
                const size_t p2 = (size_t)g.nxpp * (j + g.ny) + 2 * ii;
                vr += (sd.tau2_top * (wnl[p2] + wvr[p2])) * eps;
                vi += (sd.tau2_top * (wnl[p2 + 1] + wvr[p2 + 1])) * eps;
              }
            }
            *(double2*)(bb + (size_t)r * RS + c0) = make_double2(vr, vi);
          }
          __syncwarp();
        }
      }
      __syncthreads();
    }
  }
  double acc[R];
  if (!TC && ROLE == 3) {
    // divergence of u*: i kx u* + i ky v* + (2/h) D w*; RHS = -(div/dt) eps
    // plus the Neumann data at the walls (calcuvwt.f:87-229)
    if (live) {
      row_product16<ROLE == 3 ? 4 : 8>(sD + kk, sb + (size_t)ks * N * RS, N, acc);
      const double fac = g.hfac[ks];
      const SysDesc sd = bi.sys[s];
#pragma unroll
      for (int ci = 0; ci < NC; ++ci) {
        double vr = 0.0, vi = 0.0;
        if (cj[ci] >= 0) {
          const int j = cj[ci], ii = cii[ci];
          const size_t pr = fidx<T>(g, 2 * ii, j, k);
          const P2 u2 = *(const P2*)(F0 + pr), w2 = *(const P2*)(F1 + pr);
          const double ur = (double)u2.x, ui = (double)u2.y;
          const double wr = (double)w2.x, wi = (double)w2.y;
          const double xw = g.xw[ii], yw = g.yw[j];
          const double dr = -(xw * ui) - (yw * wi) + acc[2 * ci] * fac;
          const double di = (xw * ur) + (yw * wr) + acc[2 * ci + 1] * fac;
          vr = -((dr / dt) * eps);
          vi = -((di / dt) * eps);
          if (k == 0) {
            const size_t p1 = (size_t)g.nxpp * j + 2 * ii;
            vr -= (sd.tau1_bot * (wnl[p1] + wvr[p1])) * eps;
            vi -= (sd.tau1_bot * (wnl[p1 + 1] + wvr[p1 + 1])) * eps;
          }
          if (k == n - 1) {
            const size_t p2 = (size_t)g.nxpp * (j + g.ny) + 2 * ii;
            vr += (sd.tau2_top * (wnl[p2] + wvr[p2])) * eps;
            vi += (sd.tau2_top * (wnl[p2 + 1] + wvr[p2 + 1])) * eps;
          }
        }
        acc[2 * ci] = vr;  // column ci's divergence is no longer needed: the RHS takes its place
        acc[2 * ci + 1] = vi;
      }
    }
    __syncthreads();  // every row of w* has been read
    if (live) {
      double2* d2 = (double2*)(sb + (size_t)k * RS);
#pragma unroll
      for (int q = 0; q < R / 2; ++q) d2[q] = make_double2(acc[2 * q], acc[2 * q + 1]);
    }
    __syncthreads();
  }
  // interface system: r_e = <lvec_e, b_blk(e)>, z = M^-1 r; stored [e][r] and
  // computed with the right-hand side index fastest across lanes
  if (m > 0) {
    for (int q = tid; q < m * R; q += blockDim.x) {
      const int e = q / R, r = q - e * R;
      const int blk = e < ns - 1 ? e : e - (ns - 1) + 1;
      const double* lv = sL + (size_t)e * N;
      const double* sv = sb + (size_t)blk * N * RS + r;
      double a = 0.0;
      for (int c = 0; c < N; ++c) a += lv[c] * sv[(size_t)c * RS];
      srz[q] = a;
    }
    __syncthreads();
    for (int q = tid; q < m * R; q += blockDim.x) {
      const int e = q / R, r = q - e * R;
      const double* mr = sM + (size_t)e * m;
      double z = 0.0;
      for (int c = 0; c < m; ++c) z += mr[c] * srz[(size_t)c * R + r];
      szz[q] = z;
    }
    __syncthreads();
  }
  if constexpr (TC) {
    // x = A_ks^-1 b_ks - A_ks^-1 e_0 z_{ks-1} - A_ks^-1 e_{N-1} z_{ns-1+ks} on
    // the tensor cores; u/v, w, rho are stored, phi goes over the RHS in place
    const int gq = lane >> 2, t4 = lane & 3, MT = (N + 7) >> 3;
    for (int ks2 = wid; ks2 < ns; ks2 += nwarp) {
      double* bb = sb + (size_t)ks2 * N * RS;
      const double* blk = sA + (size_t)bi.bmap[ks2] * N * AP;
      // the pressure writes phi over its own right-hand side, half by half;
      // the other roles store to the fields and take both halves at once
      double tacc2[2][kTcMT][2];
      if (ROLE != 3) tc_block_product2(blk, AP, bb, N, lane, tacc2);
      for (int nt = 0; nt < 2; ++nt) {
        double tacc[kTcMT][2];
        if (ROLE == 3) {
          tc_block_product(blk, AP, bb, N, nt, lane, tacc);
          __syncwarp();
        } else {
#pragma unroll
          for (int mt = 0; mt < kTcMT; ++mt) {
            tacc[mt][0] = tacc2[nt][mt][0];
            tacc[mt][1] = tacc2[nt][mt][1];
          }
        }
        const int c0 = nt * 8 + 2 * t4;
#pragma unroll
        for (int mt = 0; mt < kTcMT; ++mt) {
          const int r = mt * 8 + gq;
          if (mt >= MT || r >= N) continue;
          const int kq = ks2 * N + r;
          const double p = ks2 >= 1 ? blk[r] : 0.0;
          const double q = ks2 <= ns - 2 ? blk[(size_t)(N - 1) * AP + r] : 0.0;
          double x0 = tacc[mt][0], x1 = tacc[mt][1];
          if (ks2 >= 1) {
            x0 -= p * szz[(size_t)(ks2 - 1) * R + c0];
            x1 -= p * szz[(size_t)(ks2 - 1) * R + c0 + 1];
          }
          if (ks2 <= ns - 2) {
            x0 -= q * szz[(size_t)(ns - 1 + ks2) * R + c0];
            x1 -= q * szz[(size_t)(ns - 1 + ks2) * R + c0 + 1];
          }
          if (ROLE == 3) {
            *(double2*)(bb + (size_t)r * RS + c0) = make_double2(x0, x1);
            continue;
          }
          const int ci = c0 / PER;
          if (cj[ci] < 0) continue;
          const bool second = ROLE == 0 && (c0 % 4) == 2;  // v of a u/v column
          if (ROLE == 0 && !second && meanu && cii[ci] == 0 && cj[ci] == 0) {
            x0 = meang[kq] * x0;
            x1 = meang[kq] * x1;
          }
          P2 o;
          o.x = (T)x0;
          o.y = (T)x1;
          *(P2*)((second ? F1 : F0) + fidx<T>(g, 2 * cii[ci], cj[ci], kq)) = o;
        }
        if (ROLE == 3) __syncwarp();
      }
    }
    if (ROLE != 3) return;
    // (2/h) D phi and the projection, per subdomain (phi of this warp's own
    // subdomains, written above)
    for (int ks2 = wid; ks2 < ns; ks2 += nwarp) {
      const double* bb = sb + (size_t)ks2 * N * RS;
      const double fac = g.hfac[ks2];
      for (int nt = 0; nt < 2; ++nt) {
        double tacc[kTcMT][2];
        tc_block_product(sD, AP, bb, N, nt, lane, tacc);
        const int c0 = nt * 8 + 2 * t4, ci = c0 >> 1;
        if (cj[ci] < 0) continue;
        const int j = cj[ci], ii = cii[ci];
#pragma unroll
        for (int mt = 0; mt < kTcMT; ++mt) {
          const int r = mt * 8 + gq;
          if (mt >= MT || r >= N) continue;
          const int kq = ks2 * N + r;
          const size_t pr = fidx<T>(g, 2 * ii, j, kq);
          P2 zu, zv, zw;
          if (kq < kstart) {
            zu.x = zu.y = (T)0;
            *(P2*)(F0 + pr) = zu;
            *(P2*)(F1 + pr) = zu;
            *(P2*)(F2 + pr) = zu;
            continue;
          }
          const double phr = bb[(size_t)r * RS + c0], phi = bb[(size_t)r * RS + c0 + 1];
          const P2 w2 = *(const P2*)(F2 + pr);
          double wbr = 0, wbi = 0;
          if (!(ii == 0 && j == 0)) {
            wbr = (double)w2.x - dt * (tacc[mt][0] * fac);
            wbi = (double)w2.y - dt * (tacc[mt][1] * fac);
          }
          const double dtx = dt * g.xw[ii], dty = dt * g.yw[j];
          const P2 u2 = *(const P2*)(F0 + pr), v2 = *(const P2*)(F1 + pr);
          const double ur = (double)u2.x, ui = (double)u2.y, vr = (double)v2.x, vi = (double)v2.y;
          zu.x = (T)(ur + dtx * phi);
          zu.y = (T)(ui - dtx * phr);
          zv.x = (T)(vr + dty * phi);
          zv.y = (T)(vi - dty * phr);
          zw.x = (T)wbr;
          zw.y = (T)wbi;
          *(P2*)(F0 + pr) = zu;
          *(P2*)(F1 + pr) = zv;
          *(P2*)(F2 + pr) = zw;
        }
      }
    }
    return;
  }
  // x = A_ks^-1 b_ks - A_ks^-1 e_0 z_{ks-1} - A_ks^-1 e_{N-1} z_{ns-1+ks}
  double* x = acc;  // the solution replaces the product in place
  if (live) {
    const double* col = sA + offA + (size_t)bi.bmap[ks] * N * N + kk;
    row_product16<ROLE == 3 ? 4 : 8>(col, sb + (size_t)ks * N * RS, N, acc);
    const double p = ks >= 1 ? col[0] : 0.0;
    const double q = ks <= ns - 2 ? col[(size_t)(N - 1) * N] : 0.0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      double xv = acc[r];
      if (ks >= 1) xv -= p * szz[(size_t)(ks - 1) * R + r];
      if (ks <= ns - 2) xv -= q * szz[(size_t)(ns - 1 + ks) * R + r];
      x[r] = xv;
    }
  }
  if (ROLE != 3) {
    if (ROLE == 0 && meanu && live) {
#pragma unroll
      for (int ci = 0; ci < NC; ++ci)
        if (cii[ci] == 0 && cj[ci] == 0) {
          x[PER * ci] = meang[k] * x[PER * ci];
          x[PER * ci + 1] = meang[k] * x[PER * ci + 1];
        }
    }
    if (!live) return;
#pragma unroll
    for (int ci = 0; ci < NC; ++ci) {
      if (cj[ci] < 0) continue;
      const size_t p = fidx<T>(g, 2 * cii[ci], cj[ci], k);
      const double a0 = x[PER * ci], a1 = x[PER * ci + 1];
      P2 o;
      o.x = (T)a0;
      o.y = (T)a1;
      *(P2*)(F0 + p) = o;
      if (ROLE == 0) {
        P2 o2;
        o2.x = (T)x[PER * ci + 2];
        o2.y = (T)x[PER * ci + 3];
        *(P2*)(F1 + p) = o2;
      }
    }
    return;
  }
  // pressure: phi into shared memory, (2/h) D phi, projection (calcuvwt.f:826-901)
  __syncthreads();  // every row of the RHS has been read
  if (live) {
    double2* d2 = (double2*)(sb + (size_t)k * RS);
#pragma unroll
    for (int q = 0; q < R / 2; ++q) d2[q] = make_double2(x[2 * q], x[2 * q + 1]);
  }
  __syncthreads();
  if (!live) return;
  row_product16<ROLE == 3 ? 4 : 8>(sD + kk, sb + (size_t)ks * N * RS, N, acc);
  const double fac = g.hfac[ks];
#pragma unroll
  for (int ci = 0; ci < NC; ++ci) {
    if (cj[ci] < 0) continue;
    const int j = cj[ci], ii = cii[ci];
    const size_t pr = fidx<T>(g, 2 * ii, j, k);
    P2 zu, zv, zw;
    if (k < kstart) {
      zu.x = zu.y = (T)0;
      *(P2*)(F0 + pr) = zu;
      *(P2*)(F1 + pr) = zu;
      *(P2*)(F2 + pr) = zu;
      continue;
    }
    const double phr = sb[(size_t)k * RS + 2 * ci], phi = sb[(size_t)k * RS + 2 * ci + 1];
    const P2 w2 = *(const P2*)(F2 + pr);
    double wbr = 0, wbi = 0;
    if (!(ii == 0 && j == 0)) {
      wbr = (double)w2.x - dt * (acc[2 * ci] * fac);
      wbi = (double)w2.y - dt * (acc[2 * ci + 1] * fac);
    }
    const double dtx = dt * g.xw[ii], dty = dt * g.yw[j];
    const P2 u2 = *(const P2*)(F0 + pr), v2 = *(const P2*)(F1 + pr);
    const double ur = (double)u2.x, ui = (double)u2.y, vr = (double)v2.x, vi = (double)v2.y;
    zu.x = (T)(ur + dtx * phi);
    zu.y = (T)(ui - dtx * phr);
    zv.x = (T)(vr + dty * phi);
    zv.y = (T)(vi - dty * phr);
    zw.x = (T)wbr;
    zw.y = (T)wbi;
    *(P2*)(F0 + pr) = zu;
    *(P2*)(F1 + pr) = zv;
    *(P2*)(F2 + pr) = zw;
  }
}

// ===========================================================================
// System-grouped solve with two rows per thread (u/v, w and rho).  The
// grouped solve above spends most of its time in the shared-memory pipe: each
// multiply-add of its block product takes one broadcast load of a
// right-hand-side value.  Here thread (ks, q) owns rows q and q + H of
// subdomain ks (H = ceil(N/2)), both of one inverse block, so every broadcast
// feeds two multiply-adds and the loads per multiply-add fall from 18/16 to
// 20/32.  The tables, the gather, the interface system and the order of every
// sum are those of k_solve_sys, so both give the same bits.
// ===========================================================================
constexpr int kSys2MaxThreads = 256;

// acc0/acc1[r] = sum_c col[c N (+ H)] * b[c RS + r] for two rows of one block
__device__ __forceinline__ void row_product16x2(const double* col, int H, bool has1, const double* bb, int N,
                                                double* acc0, double* acc1) {
#pragma unroll
  for (int r = 0; r < kSysR; ++r) acc0[r] = acc1[r] = 0.0;
#pragma unroll 1
  for (int c = 0; c < N; ++c) {
    const double a0 = col[(size_t)c * N];
    const double a1 = has1 ? col[(size_t)c * N + H] : 0.0;
    const double* br = bb + (size_t)c * kSysRS;
#pragma unroll
    for (int h = 0; h < kSysR; h += 8) {
      double v[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) v[r] = lds64(br + h + r);
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        acc0[h + r] += a0 * v[r];
        acc1[h + r] += a1 * v[r];
      }
    }
  }
}

template <typename T, int ROLE>
__global__ void __launch_bounds__(kSys2MaxThreads, 2) k_solve_sys2(
    Geo g, BlockInv bi, const Task* __restrict__ tasks, const int* __restrict__ col_order, T* __restrict__ F0,
    T* __restrict__ F1, double rdiv, int meanu, const double* __restrict__ meang, int* __restrict__ err) {
  static_assert(ROLE >= 0 && ROLE <= 2, "u/v, w and rho only");
  typedef typename Pair<T>::t P2;
  constexpr int R = kSysR;
  constexpr int PER = ROLE == 0 ? 4 : 2;  // right-hand sides per column
  constexpr int NC = R / PER;             // column slots
  extern __shared__ __align__(16) double sm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int cj[NC], cii[NC];
  const Task tk = tasks[blockIdx.x];
  const int n = g.nz, N = g.N, ns = g.ns, m = 2 * (ns - 1), nb = bi.nb;
  const int H = (N + 1) >> 1;
  const int tid = threadIdx.x;
  const int s = tk.sys;
  const SysSmem L = sys_smem(n, N, ns, nb, false);
  double* sA = sm + L.a;
  double* sL = sm + L.l;
  double* sM = sm + L.m;
  double* sb = sm + L.b;
  double* srz = sm + L.rz;
  double* szz = sm + L.zz;
  const uintptr_t ga = (uintptr_t)((const double*)bi.ainv + (size_t)s * nb * N * N);
  const int offA = (int)((ga & 15u) >> 3);
  const uint32_t bytesA = (uint32_t)((((size_t)nb * N * N + offA) * 8 + 15) & ~(size_t)15);
  const uint32_t bytesL = (uint32_t)((size_t)m * N * 8), bytesM = (uint32_t)((size_t)m * m * 8);
  if (tid == 0) mbar_init(&bar, 1);
  if (tid < NC) {
    const int c = tid < tk.count ? col_order[tk.first + tid] : -1;
    cj[tid] = c < 0 ? -1 : c / g.nxhp;
    cii[tid] = c < 0 ? -1 : c % g.nxhp;
  }
  __syncthreads();
  if (tid == 0) {
    mbar_expect_tx(&bar, bytesA + bytesL + bytesM);
    bulk_g2s(sA, (const void*)(ga - (uintptr_t)offA * 8), bytesA, &bar);
    if (m > 0) {
      bulk_g2s(sL, bi.lvec + (size_t)s * m * N, bytesL, &bar);
      bulk_g2s(sM, bi.minv + (size_t)s * m * m, bytesM, &bar);
    }
  }
  const double eps = bi.sys[s].eps;
  const int ks = tid / H, q0 = tid - ks * H;
  const bool live = ks < ns;
  const bool has1 = live && q0 + H < N;
  const int k0 = ks * N + q0, k1 = k0 + H;
  // gather rows k0 and k1 of every column: [row][16]
#pragma unroll 1
  for (int hr = 0; hr < 2; ++hr) {
    if (!(hr == 0 ? live : has1)) continue;
    const int k = hr == 0 ? k0 : k1;
    double v[R];
#pragma unroll
    for (int ci = 0; ci < NC; ++ci) {
      P2 a = {0, 0}, b = {0, 0};
      if (cj[ci] >= 0) {
        const size_t p = fidx<T>(g, 2 * cii[ci], cj[ci], k);
        a = *(const P2*)(F0 + p);
        if (ROLE == 0) b = *(const P2*)(F1 + p);
      }
      v[PER * ci] = (double)a.x;
      v[PER * ci + 1] = (double)a.y;
      if (ROLE == 0) {
        v[PER * ci + 2] = (double)b.x;
        v[PER * ci + 3] = (double)b.y;
      }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = -(-(v[r] / rdiv) * eps);
    double2* d2 = (double2*)(sb + (size_t)k * kSysRS);
#pragma unroll
    for (int q = 0; q < R / 2; ++q) d2[q] = make_double2(v[2 * q], v[2 * q + 1]);
  }
  const bool ok = mbar_wait(&bar, 0, 2000000000ull);
  if (__syncthreads_or(!ok)) {  // the tables never arrived: report, let the copies finish, leave
    if (tid == 0) err[1] = 1;
    mbar_wait(&bar, 0, 2000000000ull);
    return;
  }
  // interface system (the loops and sums of k_solve_sys)
  if (m > 0) {
    for (int q = tid; q < m * R; q += blockDim.x) {
      const int e = q / R, r = q - e * R;
      const int blk = e < ns - 1 ? e : e - (ns - 1) + 1;
      const double* lv = sL + (size_t)e * N;
      const double* sv = sb + (size_t)blk * N * kSysRS + r;
      double a = 0.0;
      for (int c = 0; c < N; ++c) a += lv[c] * sv[(size_t)c * kSysRS];
      srz[q] = a;
    }
    __syncthreads();
    for (int q = tid; q < m * R; q += blockDim.x) {
      const int e = q / R, r = q - e * R;
      const double* mr = sM + (size_t)e * m;
      double z = 0.0;
      for (int c = 0; c < m; ++c) z += mr[c] * srz[(size_t)c * R + r];
      szz[q] = z;
    }
    __syncthreads();
  }
  if (!live) return;
  // x = A_ks^-1 b_ks - A_ks^-1 e_0 z_{ks-1} - A_ks^-1 e_{N-1} z_{ns-1+ks}, two rows
  const double* col = sA + offA + (size_t)bi.bmap[ks] * N * N + q0;
  double acc0[R], acc1[R];
  row_product16x2(col, H, has1, sb + (size_t)ks * N * kSysRS, N, acc0, acc1);
#pragma unroll 1
  for (int hr = 0; hr < 2; ++hr) {
    if (hr == 1 && !has1) break;
    const int k = hr == 0 ? k0 : k1;
    const double* cr = col + (hr == 0 ? 0 : H);
    const double p = ks >= 1 ? cr[0] : 0.0;
    const double qv = ks <= ns - 2 ? cr[(size_t)(N - 1) * N] : 0.0;
    double x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      double xv = hr == 0 ? acc0[r] : acc1[r];
      if (ks >= 1) xv -= p * szz[(size_t)(ks - 1) * R + r];
      if (ks <= ns - 2) xv -= qv * szz[(size_t)(ns - 1 + ks) * R + r];
      x[r] = xv;
    }
    if (ROLE == 0 && meanu) {
#pragma unroll
      for (int ci = 0; ci < NC; ++ci)
        if (cii[ci] == 0 && cj[ci] == 0) {
          x[PER * ci] = meang[k] * x[PER * ci];
          x[PER * ci + 1] = meang[k] * x[PER * ci + 1];
        }
    }
#pragma unroll
    for (int ci = 0; ci < NC; ++ci) {
      if (cj[ci] < 0) continue;
      const size_t p2 = fidx<T>(g, 2 * cii[ci], cj[ci], k);
      P2 o;
      o.x = (T)x[PER * ci];
      o.y = (T)x[PER * ci + 1];
      *(P2*)(F0 + p2) = o;
      if (ROLE == 0) {
        P2 o2;
        o2.x = (T)x[PER * ci + 2];
        o2.y = (T)x[PER * ci + 3];
        *(P2*)(F1 + p2) = o2;
      }
    }
  }
}

// Distinct blocks of each system into compact storage: out[s][b] = in[s][rep[b]],
// with the Legendre filter folded in when L is given (out = L in, per column).
struct BlockRep {
  int r[IW_MAX_SUBD];
};
__global__ void k_compact_blocks(int N, int nsys, int ns, int nb, BlockRep rep, const double* __restrict__ L,
                                 const double* __restrict__ in, double* __restrict__ out) {
  const size_t nn = (size_t)N * N, tot = (size_t)nsys * nb * nn;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < tot; q += (size_t)gridDim.x * blockDim.x) {
    const size_t e = q % nn;
    const size_t sb = q / nn;
    const int b = (int)(sb % nb);
    const size_t s = sb / nb;
    const double* src = in + (s * ns + rep.r[b]) * nn;
    if (!L) {
      out[q] = src[e];
    } else {
      const int kk = (int)(e % N);
      const double* col = src + (e - kk);
      const double* lr = L + (size_t)kk * N;
      double acc = 0.0;
      for (int j = 0; j < N; ++j) acc += lr[j] * col[j];
      out[q] = acc;
    }
  }
}

// lvec[s][e][c] = sum_k A_blk^-1[k][c] v_e[k]: v_e = c_{e+1} on block e (e < ns-1),
// d_t on block t+1 (e = ns-1+t).  One thread per (system, e, c).
__global__ void k_left_vecs(Geo g, int nsys, const double* __restrict__ ainv, const double* __restrict__ cvec,
                            const double* __restrict__ dvec, double* __restrict__ lvec) {
  const int N = g.N, ns = g.ns, m = 2 * (ns - 1);
  const size_t tot = (size_t)nsys * m * N;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < tot; q += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(q % N);
    const int e = (int)((q / N) % m);
    const size_t s = q / ((size_t)N * m);
    int blk;
    const double* v;
    if (e < ns - 1) {
      blk = e;
      v = cvec + (s * ns + e + 1) * N;
    } else {
      blk = e - (ns - 1) + 1;
      v = dvec + (s * ns + blk - 1) * N;
    }
    const double* ai = ainv + (s * ns + blk) * (size_t)N * N + (size_t)c * N;
    double acc = 0.0;
    for (int k = 0; k < N; ++k) acc += ai[k] * v[k];
    lvec[q] = acc;
  }
}

// ===========================================================================
// Interface averaging (penalty.f:714-775).
// ===========================================================================
// apply the round-trip projection P in place to all planes except the
// interface planes (km, k of every interface), which go through real
// transforms instead.  Thread per (j, k, field) for the kx=0 pair and the
// Nyquist column.
template <typename T>
__global__ void k_project_planes(Geo g, T* F0, T* F1, T* F2, T* F3, int skip_iface) {
  // grid: x over y rows, y over z levels, z over the 4 fields (32-bit indices)
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= g.ny) return;
  const int k = blockIdx.y, q = blockIdx.z;
  if (skip_iface) {
    int kl = k % g.N;
    if ((kl == 0 && k > 0) || (kl == g.N - 1 && k < g.nz - 1)) return;
  }
  T* F = q == 0 ? F0 : q == 1 ? F1 : q == 2 ? F2 : F3;
  int jp = (g.ny - j) % g.ny;
  // Nyquist: independent per j
  size_t pn = fidx<T>(g, g.nx, j, k);
  F[pn] = F[pn] * (T)g.scaley;
  F[pn + 1] = 0;
  if (j <= jp) {
    size_t pa = fidx<T>(g, 0, j, k), pb = fidx<T>(g, 0, jp, k);
    T ar = F[pa], ai = F[pa + 1], br = F[pb], bi = F[pb + 1];
    T nr = (T)0.5 * (ar + br), ni = (T)0.5 * (ai - bi);
    F[pa] = nr;
    F[pa + 1] = ni;
    if (jp != j) {
      F[pb] = nr;
      F[pb + 1] = -ni;
    }
  }
}

// gather the 4 planes around each interface into a compact buffer:
// G[(q*(ns-1)+f)*4 + m] plane = F_q level (f+1)*N - 2 + m; back: add the
// averaging change held in G to the two interface planes.
// Grid: x over the points of a plane, y over the 16 (ns - 1) planes (no
// 64-bit division per element).
template <typename T>
__global__ void k_iface_gather(Geo g, const T* F0, const T* F1, const T* F2, const T* F3, T* G, int back) {
  const size_t per = g.plane;
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= per) return;
  const int pl = blockIdx.y;
  int m = pl % 4;
  int f = (pl / 4) % (g.ns - 1);
  int q = pl / (4 * (g.ns - 1));
  int k = (f + 1) * g.N - 2 + m;
  const T* F = q == 0 ? F0 : q == 1 ? F1 : q == 2 ? F2 : F3;
  if (!back) {
    G[(size_t)pl * per + e] = F[(size_t)k * per + e];
  } else if (m == 1 || m == 2) {
    ((T*)F)[(size_t)k * per + e] += G[(size_t)pl * per + e];  // spectral change made by the averaging
  }
}

// per (row j, interface plane group): x-inverse of 4 rows, average, x-forward
// of the change of the 2 interface rows.
template <typename T>
__global__ void k_iface_rows(Geo g, T* G, FftPlan pl, const typename cplx_t<T>::type* __restrict__ Wm,
                             const typename cplx_t<T>::type* __restrict__ Wn, int* counts) {
  typedef typename cplx_t<T>::type C;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int M = g.nx / 2, nx = g.nx;
  C* A = (C*)smraw;
  C* B = A + 4 * M;
  const int j = blockIdx.x;
  const int grp = blockIdx.y;  // q*(ns-1)+f
  const int q = grp / (g.ns - 1);
  const size_t per = g.plane;
  for (int m = 0; m < 4; ++m)
    xinv_prep<C, T>(G + (size_t)(grp * 4 + m) * per + (size_t)j * g.nxpp, A + m * M, M, Wn, 0, (T)0, threadIdx.x,
                    blockDim.x);
  __syncthreads();
  C* ph = fft_run<C>(A, B, pl, 4, Wm, true, threadIdx.x, blockDim.x);
  T* P = (T*)ph;
  int cnt = 0;
  // The interface rows become the change made by the averaging (0 where it
  // does not trigger): the spectral planes are then P(F) + transform of the
  // change, so points left alone never take the round trip's rounding.
  for (int i = threadIdx.x; i < nx; i += blockDim.x) {
    T fsp = P[2 * nx + i], fsm = P[1 * nx + i];
    T favg2 = fsp + fsm;
    T c0 = fabs(fsp - fsm) / fabs(favg2);
    T d1 = 0, d2 = 0;
    if (c0 > (T)0.005) {
      T ff = P[0 * nx + i] * (T)0.5 + P[1 * nx + i] * (T)0 + P[2 * nx + i] * (T)0 + P[3 * nx + i] * (T)0.5;
      d1 = ff - fsm;
      d2 = ff - fsp;
      ++cnt;
    }
    P[1 * nx + i] = d1;
    P[2 * nx + i] = d2;
  }
  if (cnt) atomicAdd(counts + q, cnt);
  __syncthreads();
  C* other = (ph == A) ? B : A;
  C* sp = fft_run<C>(ph + M, other + M, pl, 2, Wm, false, threadIdx.x, blockDim.x);
  const T invN = (T)1 / (T)nx;
  for (int t = threadIdx.x; t < 2 * (M + 1); t += blockDim.x) {
    int m = t / (M + 1), kk = t % (M + 1);
    C v = xfwd_post<C>(sp + m * M, kk, M, Wn, invN);
    T* p = G + (size_t)(grp * 4 + 1 + m) * per + (size_t)j * g.nxpp + 2 * kk;
    p[0] = v.x;
    p[1] = v.y;
  }
}

// ===========================================================================
// generic whole-field helpers for the Fortran-style entry points
// ===========================================================================
template <typename T>
__global__ void k_xfft_field(Geo g, T* F, int nk, int inv, FftPlan pl, const typename cplx_t<T>::type* __restrict__ Wm,
                             const typename cplx_t<T>::type* __restrict__ Wn) {
  typedef typename cplx_t<T>::type C;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int M = g.nx / 2, nx = g.nx;
  C* A = (C*)smraw;
  C* B = A + M;
  const int row = blockIdx.x;  // j + ny*k
  T* rp = F + (size_t)row * g.nxpp;
  if (inv) {
    xinv_prep<C, T>(rp, A, M, Wn, 0, (T)0, threadIdx.x, blockDim.x);
    __syncthreads();
    C* r = fft_run<C>(A, B, pl, 1, Wm, true, threadIdx.x, blockDim.x);
    T* P = (T*)r;
    for (int i = threadIdx.x; i < g.nxpp; i += blockDim.x) rp[i] = i < nx ? P[i] : (T)0;
  } else {
    for (int i = threadIdx.x; i < M; i += blockDim.x) A[i] = cmk<C>(rp[2 * i], rp[2 * i + 1]);
    __syncthreads();
    C* r = fft_run<C>(A, B, pl, 1, Wm, false, threadIdx.x, blockDim.x);
    const T invN = (T)1 / (T)nx;
    for (int t = threadIdx.x; t < M + 1; t += blockDim.x) {
      C v = xfwd_post<C>(r, t, M, Wn, invN);
      // write after everyone has read r: r is a different buffer than rp
      rp[2 * t] = v.x;
      rp[2 * t + 1] = v.y;
    }
  }
}

template <typename T>
__global__ void k_mulikx(Geo g, T* F) {
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long)(g.ntot / 2)) return;
  size_t p = 2 * (size_t)gid;
  int ii = (int)((p % g.nxpp) / 2);
  T kx = (T)g.xw[ii];
  T a = F[p], b = F[p + 1];
  F[p] = -(kx * b);
  F[p + 1] = kx * a;
}

template <typename T>
__global__ void k_dz_field(Geo g, const T* __restrict__ a, T* __restrict__ b) {
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long)g.ntot) return;
  size_t e = gid % g.plane;
  int k = gid / g.plane;
  int ks = k / g.N, k1 = k % g.N;
  double s = 0.0;
  for (int k2 = 0; k2 < g.N; ++k2) s += g.D[k1 * g.N + k2] * (double)a[(size_t)(ks * g.N + k2) * g.plane + e];
  b[gid] = (T)(s * g.hfac[ks]);
}

// filter_3dlegenfourier on a spectral field, in place
template <typename T>
__global__ void k_filter_field(Geo g, T* F, int ifourier, int ilegen) {
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long total = (long)g.nxpp * g.ny * g.ns;
  if (gid >= total) return;
  int i = gid % g.nxpp;
  long r = gid / g.nxpp;
  int j = r % g.ny;
  int ks = r / g.ny;
  const int N = g.N;
  double v[kMaxN];
  double cf = ifourier ? g.cfour[(size_t)j * g.nxhp + (i >> 1)] : 1.0;
  for (int k = 0; k < N; ++k) v[k] = (double)F[fidx<T>(g, i, j, ks * N + k)] * cf;
  for (int k1 = 0; k1 < N; ++k1) {
    double s = 0;
    if (ilegen)
      for (int k2 = 0; k2 < N; ++k2) s += g.Lfil[k1 * N + k2] * v[k2];
    else
      s = v[k1];
    F[fidx<T>(g, i, j, ks * N + k1)] = (T)s;
  }
}

// reductions for diagnostics: physical-space sums over i<nx, k>=1
// Deterministic: a fixed grid and stride, fixed-order warp and block sums,
// and each block adds its sum to its own slot part[blockIdx.x]; the host adds
// the slots in order.  Repeated calls on the same state give the same bits.
template <typename T>
__global__ void k_reduce_sq(Geo g, const T* __restrict__ a, int kmin, double* part) {
  __shared__ double ws[32];
  double s = 0;
  long total = (long)g.nx * g.ny * (g.nz - kmin);
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    int i = t % g.nx;
    long r = t / g.nx;
    int j = r % g.ny;
    int k = kmin + r / g.ny;
    double x = (double)a[fidx<T>(g, i, j, k)];
    s += x * x;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b += ws[w];
    part[blockIdx.x] += b;
  }
}

// maxcalc statistics of one physical field (various.f:665-987 without the
// adaptive step): extrema starting from the reference's initial values (0, or
// 1 for rho whose background 1 + rhograd z is added), the CFL maximum
// (x, y: |f| dt/dx; z: |w| dt/dz with the reference's merged-interface
// spacing, dzinv), and for w the sum of squares and count below zlim.
// Per-block partials: part[5*block + {min, max, cfl, sum w^2, count}].
template <typename T>
__global__ void k_phys_stats(Geo g, const T* __restrict__ a, int q, const double* __restrict__ zg,
                             const double* __restrict__ dzinv, double cflh, double rg, double zlim, double* part) {
  double mn = q == 3 ? 1.0 : 0.0, mx = 0.0, cf = 0.0, s2 = 0.0, cnt = 0.0;
  const long total = (long)g.nx * g.ny * g.nz;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const int i = (int)(t % g.nx);
    const long r = t / g.nx;
    const int j = (int)(r % g.ny), k = (int)(r / g.ny);
    double x = (double)a[fidx<T>(g, i, j, k)];
    if (q == 0 || q == 1) cf = fmax(cf, fabs(x) * cflh);
    if (q == 2) {
      cf = fmax(cf, fabs(x) * g.dt * dzinv[k]);
      if (zg[k] < zlim) {
        s2 += x * x;
        cnt += 1.0;
      }
    }
    if (q == 3) x += 1.0 + rg * zg[k];
    mn = fmin(mn, x);
    mx = fmax(mx, x);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    cf = fmax(cf, __shfl_xor_sync(0xffffffffu, cf, o));
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  }
  __shared__ double sh[32][5];
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    sh[w][0] = mn;
    sh[w][1] = mx;
    sh[w][2] = cf;
    sh[w][3] = s2;
    sh[w][4] = cnt;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int v = 1; v < nw; ++v) {
      mn = fmin(mn, sh[v][0]);
      mx = fmax(mx, sh[v][1]);
      cf = fmax(cf, sh[v][2]);
      s2 += sh[v][3];
      cnt += sh[v][4];
    }
    double* o = part + 5 * (size_t)blockIdx.x;
    o[0] = mn;
    o[1] = mx;
    o[2] = cf;
    o[3] = s2;
    o[4] = cnt;
  }
}

template <typename T>
__global__ void k_nonfinite(const T* __restrict__ a, size_t n, int* flag) {
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
    if (!isfinite((double)a[t])) {
      atomicExch(flag, 1);
      return;
    }
}

template <typename T, typename U>
__global__ void k_convert(const T* __restrict__ a, U* __restrict__ b, size_t n) {
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
    b[t] = (U)a[t];
}

#include "iw_host.inl"
