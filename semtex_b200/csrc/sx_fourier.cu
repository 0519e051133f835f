// sx_fourier.cu -- z-direction (Fourier) transform of field planes.
//
// semtex's dDFTr (femlib/fourier.c:47-171) as used by AuxField::transform
// (src/auxfield.cpp:1133-1170): nz real planes of a field, point p of plane
// z at data[z * stride + p], transformed along z at every point.
//   forward (sign = +1): X_k = (1/nz) sum_j x_j exp(-2 pi i j k / nz) --
//     the sign of DMPFFT's call of DGPFA with ISIGN = -1
//     (femlib/temfftd.F:218-238) and dDFTr's 1/tlen scaling -- stored as
//     plane 0 = Re X_0, plane 1 = Re X_{nz/2} (the Nyquist datum), planes
//     2k, 2k+1 = Re X_k, Im X_k for k = 1 .. nz/2 - 1 (fourier.c:58-63);
//   inverse (sign = -1): x_j = X_0 + (-1)^j X_{nz/2} + 2 sum_{k=1}^{nz/2-1}
//     Re(X_k exp(+2 pi i j k / nz)), unscaled, so that inverse(forward(x))
//     = x.
// Lengths 2, 4, ..., 64 (config 2 uses 64): one pass, k_z_fwd / k_z_inv;
// 128, 256, 512: one pass through shared memory, k_z_fwd_s / k_z_inv_s.
// A thread holds one point's whole z-line in registers: the real transform
// of length N is a complex FFT of length M = N/2 on z_m = x_2m + i x_2m+1
// (radix-2, decimation in time, every index a compile-time constant), then
// the split X_k = E_k + W^k O_k with E_k = (Z_k + conj Z_{M-k})/2, O_k =
// (Z_k - conj Z_{M-k})/2i, W = exp(-2 pi i / N); the inverse runs the same
// steps backwards.  A warp's loads and stores of one plane are 32
// consecutive doubles; the field is read once and written once.  Other
// lengths: cuFFT's batched real transform (one transform per point, element
// stride = the plane stride, loaded on first use) into a half-spectrum
// workspace [nz/2 + 1][npts], and this file's packing kernels.
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <vector>
#include <map>
#include <mutex>
#include <tuple>

#include <cufft.h>

#include "sx_internal.h"

namespace sx {

namespace {

// cuFFT entry points, resolved from the shared library at first use.
struct CufftApi {
  decltype(&cufftPlanMany) planMany = nullptr;
  decltype(&cufftSetStream) setStream = nullptr;
  decltype(&cufftExecD2Z) execD2Z = nullptr;
  decltype(&cufftExecZ2D) execZ2D = nullptr;
  decltype(&cufftDestroy) destroy = nullptr;
  bool ok = false;
};

const CufftApi &cufft_api() {
  static CufftApi api;
  static std::once_flag once;
  std::call_once(once, []() {
    void *h = dlopen("libcufft.so.11", RTLD_NOW | RTLD_LOCAL);
    if (!h) h = dlopen("libcufft.so", RTLD_NOW | RTLD_LOCAL);
    if (!h) return;
    api.planMany = reinterpret_cast<decltype(&cufftPlanMany)>(dlsym(h, "cufftPlanMany"));
    api.setStream = reinterpret_cast<decltype(&cufftSetStream)>(dlsym(h, "cufftSetStream"));
    api.execD2Z = reinterpret_cast<decltype(&cufftExecD2Z)>(dlsym(h, "cufftExecD2Z"));
    api.execZ2D = reinterpret_cast<decltype(&cufftExecZ2D)>(dlsym(h, "cufftExecZ2D"));
    api.destroy = reinterpret_cast<decltype(&cufftDestroy)>(dlsym(h, "cufftDestroy"));
    api.ok = api.planMany && api.setStream && api.execD2Z && api.execZ2D && api.destroy;
  });
  return api;
}

// Plans and workspaces per (device, nz, npts, stride, direction), kept for
// the life of the process (a plan is a few kB; the workspace is the
// half-spectrum).
struct ZPlan {
  cufftHandle plan = 0;
  DBuf<double2> spec;  // [nz/2 + 1][npts]
};
std::mutex g_mu;
std::map<std::tuple<int, int, int, int, int>, std::unique_ptr<ZPlan>> g_plans;

bool factors_235(int n) {
  for (int f : {2, 3, 5})
    while (n % f == 0) n /= f;
  return n == 1;
}

}  // namespace

// exp(-2 pi i t / TWN), t = 0 .. TWN/2, from the host's cos / sin in FP64;
// a length-L stage uses t = j * (TWN / L).
constexpr int TWN = 512;
__constant__ double c_twr[TWN / 2 + 1], c_twi[TWN / 2 + 1];

static int ensure_twiddles() {
  static std::mutex mu;
  static std::vector<char> done(256, 0);
  int dev = 0;
  SX_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 256 && done[dev]) return SX_OK;
  double wr[TWN / 2 + 1], wi[TWN / 2 + 1];
  for (int t = 0; t <= TWN / 2; t++) {
    const double a = 2.0 * M_PI * t / TWN;
    wr[t] = std::cos(a);
    wi[t] = -std::sin(a);
  }
  wr[TWN / 4] = 0.0;  // exact at the quarter and half turns
  wi[TWN / 4] = -1.0;
  wr[TWN / 2] = -1.0;
  wi[TWN / 2] = 0.0;
  SX_CUDA(cudaMemcpyToSymbol(c_twr, wr, sizeof(wr)));
  SX_CUDA(cudaMemcpyToSymbol(c_twi, wi, sizeof(wi)));
  if (dev < 256) done[dev] = 1;
  return SX_OK;
}

constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n / 2); }
constexpr int bitrev(int v, int bits) {
  int r = 0;
  for (int b = 0; b < bits; b++) {
    r = (r << 1) | (v & 1);
    v >>= 1;
  }
  return r;
}

// One radix-2 stage (butterflies of span LEN) of an in-place decimation-in-
// time FFT of length M, then the next stage; INV conjugates the twiddles.
// Stages are template instances so that every register index is a
// compile-time constant.
template <int M, int LEN, bool INV>
struct FftStage {
  static __device__ __forceinline__ void run(double (&re)[M], double (&im)[M]) {
#pragma unroll
    for (int i = 0; i < M; i += LEN) {
#pragma unroll
      for (int j = 0; j < LEN / 2; j++) {
        const int t = j * (TWN / LEN);
        const double wr = c_twr[t], wi = INV ? -c_twi[t] : c_twi[t];
        const int a = i + j, b = i + j + LEN / 2;
        const double vr = re[b] * wr - im[b] * wi, vi = re[b] * wi + im[b] * wr;
        re[b] = re[a] - vr;
        im[b] = im[a] - vi;
        re[a] += vr;
        im[a] += vi;
      }
    }
    FftStage<M, LEN * 2, INV>::run(re, im);
  }
};
template <int M, bool INV>
struct FftStage<M, M * 2, INV> {
  static __device__ __forceinline__ void run(double (&)[M], double (&)[M]) {}
};

// In-place radix-2 FFT of length M on bit-reversed input, natural-order
// output, unscaled.
template <int M, bool INV>
__device__ __forceinline__ void cfft_reg(double (&re)[M], double (&im)[M]) {
  FftStage<M, 2, INV>::run(re, im);
}

template <int N>
__global__ void __launch_bounds__(128) k_z_fwd(double *__restrict__ data, int npts, long long stride, double scale) {
  constexpr int M = N / 2, LB = ilog2c(M);
  const int p = blockIdx.x * 128 + threadIdx.x;
  if (p >= npts) return;
  double re[M], im[M];
#pragma unroll
  for (int m = 0; m < M; m++) {
    re[bitrev(m, LB)] = data[(2 * m) * stride + p];
    im[bitrev(m, LB)] = data[(2 * m + 1) * stride + p];
  }
  cfft_reg<M, false>(re, im);
  // k = 0: E_0 = Re Z_0, O_0 = Im Z_0; X_0 = E_0 + O_0, X_M = E_0 - O_0
  data[p] = (re[0] + im[0]) * scale;
  data[stride + p] = (re[0] - im[0]) * scale;
#pragma unroll
  for (int k = 1; k < M; k++) {
    const double yr = re[M - k], yi = -im[M - k];  // conj Z_{M-k}
    const double er = 0.5 * (re[k] + yr), ei = 0.5 * (im[k] + yi);
    const double orr = 0.5 * (im[k] - yi), oi = -0.5 * (re[k] - yr);  // (Z_k - conj Z_{M-k}) / 2i
    const int t = k * (TWN / N);
    const double wr = c_twr[t], wi = c_twi[t];
    data[(2 * k) * stride + p] = (er + (orr * wr - oi * wi)) * scale;
    data[(2 * k + 1) * stride + p] = (ei + (orr * wi + oi * wr)) * scale;
  }
}

template <int N>
__global__ void __launch_bounds__(128) k_z_inv(double *__restrict__ data, int npts, long long stride) {
  constexpr int M = N / 2, LB = ilog2c(M);
  const int p = blockIdx.x * 128 + threadIdx.x;
  if (p >= npts) return;
  double re[M], im[M];
  {
    // k = 0: E_0 = (X_0 + X_M)/2, O_0 = (X_0 - X_M)/2, Z_0 = E_0 + i O_0
    const double x0 = data[p], xm = data[stride + p];
    re[0] = 0.5 * (x0 + xm);
    im[0] = 0.5 * (x0 - xm);
  }
  // E_k = (X_k + conj X_{M-k})/2, O_k = (X_k - conj X_{M-k}) conj(W^k)/2,
  // Z_k = E_k + i O_k, for k and M - k together
#pragma unroll
  for (int k = 1; k <= M / 2; k++) {
    const int kk = M - k;
    const double ar = data[(2 * k) * stride + p], ai = data[(2 * k + 1) * stride + p];
    const double br = data[(2 * kk) * stride + p], bi = data[(2 * kk + 1) * stride + p];
#pragma unroll
    for (int side = 0; side < (k == kk ? 1 : 2); side++) {
      const int q = side ? kk : k;
      const double xr = side ? br : ar, xi = side ? bi : ai;   // X_q
      const double cr = side ? ar : br, ci = side ? -ai : -bi;  // conj X_{M-q}
      const double er = 0.5 * (xr + cr), ei = 0.5 * (xi + ci);
      const double dr = 0.5 * (xr - cr), di = 0.5 * (xi - ci);
      const int t = q * (TWN / N);
      const double wr = c_twr[t], wi = -c_twi[t];  // conj W^q
      const double orr = dr * wr - di * wi, oi = dr * wi + di * wr;
      re[bitrev(q, LB)] = er - oi;  // E + i O
      im[bitrev(q, LB)] = ei + orr;
    }
  }
  cfft_reg<M, true>(re, im);
#pragma unroll
  for (int m = 0; m < M; m++) {
    data[(2 * m) * stride + p] = 2.0 * re[m];
    data[(2 * m + 1) * stride + p] = 2.0 * im[m];
  }
}

// Lengths 128, 256, 512: a block of eight warps takes 32 points (lane =
// point); the half-length complex sequence z (length M = N/2) of each point
// lies in shared memory, Zr/Zi[m][32], in natural order.  The complex FFT
// of length M = M1 M2 runs in four steps with m = M2 m1 + m2 and
// k = k1 + M1 k2: (1) the M2 FFTs of length M1 over m1, each a warp's, in
// registers; (2) the twiddles W_M^(m2 k1); (3) the M1 FFTs of length M2
// over m2, in registers.  Two round trips through shared memory and two
// barriers, against one per radix-2 stage (log2 M).  Z_k ends at row
// M2 (k mod M1) + k / M1.  The real-to-complex steps around it are the
// register kernels'; loads and stores of a plane are 32 consecutive doubles.
constexpr size_t zsmem(int nz) { return (size_t)nz * 32 * sizeof(double); }
constexpr int ZW = 8;  // warps a block: every sub-FFT of a pass at once

template <int M>
struct FourStep {
  static constexpr int M1 = M >= 128 ? 16 : 8, M2 = M / M1;
  static __device__ __forceinline__ int row(int k) { return M2 * (k % M1) + k / M1; }
};

// W_M^e = exp(-2 pi i e / M) from the half-turn table (conjugated for the
// inverse).
template <int M>
__device__ __forceinline__ void twiddle(int e, bool inv, double &wr, double &wi) {
  e &= M - 1;
  const bool neg = e >= M / 2;
  const int t = (neg ? e - M / 2 : e) * (TWN / M);
  wr = neg ? -c_twr[t] : c_twr[t];
  wi = neg ? -c_twi[t] : c_twi[t];
  if (inv) wi = -wi;
}

template <int M, bool INV>
__device__ __forceinline__ void four_step(double *Zr, double *Zi) {
  using F = FourStep<M>;
  constexpr int M1 = F::M1, M2 = F::M2, L1 = ilog2c(M1), L2 = ilog2c(M2);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;  // ZW warps
  for (int m2 = w; m2 < M2; m2 += ZW) {
    double re[M1], im[M1];
#pragma unroll
    for (int m1 = 0; m1 < M1; m1++) {
      re[bitrev(m1, L1)] = Zr[(M2 * m1 + m2) * 32 + lane];
      im[bitrev(m1, L1)] = Zi[(M2 * m1 + m2) * 32 + lane];
    }
    cfft_reg<M1, INV>(re, im);
#pragma unroll
    for (int k1 = 0; k1 < M1; k1++) {
      double wr, wi;
      twiddle<M>(m2 * k1, INV, wr, wi);
      const double xr = re[k1] * wr - im[k1] * wi, xi = re[k1] * wi + im[k1] * wr;
      Zr[(M2 * k1 + m2) * 32 + lane] = xr;
      Zi[(M2 * k1 + m2) * 32 + lane] = xi;
    }
  }
  __syncthreads();
  for (int k1 = w; k1 < M1; k1 += ZW) {
    double re[M2], im[M2];
#pragma unroll
    for (int m2 = 0; m2 < M2; m2++) {
      re[bitrev(m2, L2)] = Zr[(M2 * k1 + m2) * 32 + lane];
      im[bitrev(m2, L2)] = Zi[(M2 * k1 + m2) * 32 + lane];
    }
    cfft_reg<M2, INV>(re, im);
#pragma unroll
    for (int k2 = 0; k2 < M2; k2++) {
      Zr[(M2 * k1 + k2) * 32 + lane] = re[k2];
      Zi[(M2 * k1 + k2) * 32 + lane] = im[k2];
    }
  }
  __syncthreads();
}

template <int N>
__global__ void __launch_bounds__(ZW * 32, 3) k_z_fwd_s(double *__restrict__ data, int npts, long long stride,
                                                  double scale) {
  constexpr int M = N / 2;
  using F = FourStep<M>;
  extern __shared__ __align__(16) double zs[];
  double *Zr = zs, *Zi = zs + M * 32;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;  // ZW warps
  const int p = blockIdx.x * 32 + lane;
  const bool ok = p < npts;
#pragma unroll 4
  for (int m = w; m < M; m += ZW) {
    Zr[m * 32 + lane] = ok ? data[(2 * m) * stride + p] : 0.0;
    Zi[m * 32 + lane] = ok ? data[(2 * m + 1) * stride + p] : 0.0;
  }
  __syncthreads();
  four_step<M, false>(Zr, Zi);
  if (!ok) return;  // no barrier follows
#pragma unroll 2
  for (int k = w; k <= M / 2; k += ZW) {
    if (k == 0) {
      const int r0 = F::row(0);
      data[p] = (Zr[r0 * 32 + lane] + Zi[r0 * 32 + lane]) * scale;
      data[stride + p] = (Zr[r0 * 32 + lane] - Zi[r0 * 32 + lane]) * scale;
      continue;
    }
    // X_k from Z_k and conj Z_{M-k}; and X_{M-k} from the same pair
    const int kk = M - k, rk = F::row(k), rkk = F::row(kk);
    const double zr = Zr[rk * 32 + lane], zi = Zi[rk * 32 + lane];
    const double qr = Zr[rkk * 32 + lane], qi = Zi[rkk * 32 + lane];
    for (int side = 0; side < (k == kk ? 1 : 2); side++) {
      const int q = side ? kk : k;
      const double ar = side ? qr : zr, ai = side ? qi : zi;   // Z_q
      const double yr = side ? zr : qr, yi = side ? -zi : -qi;  // conj Z_{M-q}
      const double er = 0.5 * (ar + yr), ei = 0.5 * (ai + yi);
      const double orr = 0.5 * (ai - yi), oi = -0.5 * (ar - yr);
      const int t = q * (TWN / N);
      const double wr = c_twr[t], wi = c_twi[t];
      data[(2 * q) * stride + p] = (er + (orr * wr - oi * wi)) * scale;
      data[(2 * q + 1) * stride + p] = (ei + (orr * wi + oi * wr)) * scale;
    }
  }
}

template <int N>
__global__ void __launch_bounds__(ZW * 32, 3) k_z_inv_s(double *__restrict__ data, int npts, long long stride) {
  constexpr int M = N / 2;
  using F = FourStep<M>;
  extern __shared__ __align__(16) double zs[];
  double *Zr = zs, *Zi = zs + M * 32;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;  // ZW warps
  const int p = blockIdx.x * 32 + lane;
  const bool ok = p < npts;
#pragma unroll 2
  for (int k = w; k <= M / 2; k += ZW) {
    if (k == 0) {
      const double x0 = ok ? data[p] : 0.0, xm = ok ? data[stride + p] : 0.0;
      Zr[0 * 32 + lane] = 0.5 * (x0 + xm);
      Zi[0 * 32 + lane] = 0.5 * (x0 - xm);
      continue;
    }
    const int kk = M - k;
    const double ar = ok ? data[(2 * k) * stride + p] : 0.0, ai = ok ? data[(2 * k + 1) * stride + p] : 0.0;
    const double br = ok ? data[(2 * kk) * stride + p] : 0.0, bi = ok ? data[(2 * kk + 1) * stride + p] : 0.0;
    for (int side = 0; side < (k == kk ? 1 : 2); side++) {
      const int q = side ? kk : k;
      const double xr = side ? br : ar, xi = side ? bi : ai;
      const double cr = side ? ar : br, ci = side ? -ai : -bi;
      const double er = 0.5 * (xr + cr), ei = 0.5 * (xi + ci);
      const double dr = 0.5 * (xr - cr), di = 0.5 * (xi - ci);
      const int t = q * (TWN / N);
      const double wr = c_twr[t], wi = -c_twi[t];
      const double orr = dr * wr - di * wi, oi = dr * wi + di * wr;
      Zr[q * 32 + lane] = er - oi;
      Zi[q * 32 + lane] = ei + orr;
    }
  }
  __syncthreads();
  four_step<M, true>(Zr, Zi);
  if (!ok) return;
#pragma unroll 4
  for (int m = w; m < M; m += ZW) {
    const int r = F::row(m);
    data[(2 * m) * stride + p] = 2.0 * Zr[r * 32 + lane];
    data[(2 * m + 1) * stride + p] = 2.0 * Zi[r * 32 + lane];
  }
}

template <int N>
static int launch_smem(double *d, int npts, long long stride, int sign, cudaStream_t st) {
  static std::once_flag once;
  static cudaError_t attr = cudaSuccess;
  std::call_once(once, []() {
    attr = cudaFuncSetAttribute(k_z_fwd_s<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zsmem(N));
    if (attr == cudaSuccess)
      attr = cudaFuncSetAttribute(k_z_inv_s<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zsmem(N));
  });
  SX_CUDA(attr);
  const int grid = (npts + 31) / 32;
  if (sign == 1)
    k_z_fwd_s<N><<<grid, ZW * 32, zsmem(N), st>>>(d, npts, stride, 1.0 / N);
  else
    k_z_inv_s<N><<<grid, ZW * 32, zsmem(N), st>>>(d, npts, stride);
  return SX_OK;
}

template <int N>
static void launch_reg(double *d, int npts, long long stride, int sign, cudaStream_t st) {
  const int grid = (npts + 127) / 128;
  if (sign == 1)
    k_z_fwd<N><<<grid, 128, 0, st>>>(d, npts, stride, 1.0 / N);
  else
    k_z_inv<N><<<grid, 128, 0, st>>>(d, npts, stride);
}

// spec[k][p] (k = 0 .. nz/2) -> data planes in semtex order, times 1/nz.
__global__ void k_z_pack(const double2 *__restrict__ spec, double *__restrict__ data, int nz, int npts,
                         long long stride, double scale) {
  const int nh = nz / 2;
  const long long n = (long long)(nh + 1) * npts;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i / npts), p = (int)(i - (long long)k * npts);
    const double2 v = spec[i];
    if (k == 0) {
      data[p] = v.x * scale;
    } else if (k == nh) {
      data[stride + p] = v.x * scale;
    } else {
      data[(2 * k) * stride + p] = v.x * scale;
      data[(2 * k + 1) * stride + p] = v.y * scale;
    }
  }
}

// data planes in semtex order -> spec[k][p] (Hermitian half spectrum, the
// imaginary parts of modes 0 and nz/2 zero).
__global__ void k_z_unpack(const double *__restrict__ data, double2 *__restrict__ spec, int nz, int npts,
                           long long stride) {
  const int nh = nz / 2;
  const long long n = (long long)(nh + 1) * npts;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i / npts), p = (int)(i - (long long)k * npts);
    double2 v;
    if (k == 0)
      v = make_double2(data[p], 0.0);
    else if (k == nh)
      v = make_double2(data[stride + p], 0.0);
    else
      v = make_double2(data[(2 * k) * stride + p], data[(2 * k + 1) * stride + p]);
    spec[i] = v;
  }
}

}  // namespace sx

using namespace sx;

extern "C" int sx_transform_z(double *d_data, int nz, int plane_stride, int npts, int sign, void *stream) {
  if (!d_data || nz < 1 || plane_stride <= 0 || npts < 0 || npts > plane_stride || (sign != 1 && sign != -1))
    return SX_ERR_ARG;
  if (nz == 1 || npts == 0) return SX_OK;  // a 2-D field: nothing to transform
  if (nz % 2 || !factors_235(nz)) {
    set_error("transform length %d: needs an even length with prime factors 2, 3, 5 (fourier.c:135-143)", nz);
    return SX_ERR_ARG;
  }
  if (nz <= 64 && (nz & (nz - 1)) == 0) {
    // one pass in registers, enqueued without waiting (no workspace)
    SX_TRY(ensure_twiddles());
    cudaStream_t st = (cudaStream_t)stream;
    switch (nz) {
      case 2: launch_reg<2>(d_data, npts, plane_stride, sign, st); break;
      case 4: launch_reg<4>(d_data, npts, plane_stride, sign, st); break;
      case 8: launch_reg<8>(d_data, npts, plane_stride, sign, st); break;
      case 16: launch_reg<16>(d_data, npts, plane_stride, sign, st); break;
      case 32: launch_reg<32>(d_data, npts, plane_stride, sign, st); break;
      default: launch_reg<64>(d_data, npts, plane_stride, sign, st); break;
    }
    SX_CUDA(cudaGetLastError());
    return SX_OK;
  }
  if (nz <= TWN && (nz & (nz - 1)) == 0) {
    // one pass through shared memory, enqueued without waiting
    SX_TRY(ensure_twiddles());
    cudaStream_t st = (cudaStream_t)stream;
    switch (nz) {
      case 128: SX_TRY(launch_smem<128>(d_data, npts, plane_stride, sign, st)); break;
      case 256: SX_TRY(launch_smem<256>(d_data, npts, plane_stride, sign, st)); break;
      default: SX_TRY(launch_smem<512>(d_data, npts, plane_stride, sign, st)); break;
    }
    SX_CUDA(cudaGetLastError());
    return SX_OK;
  }
  const CufftApi &api = cufft_api();
  if (!api.ok) {
    set_error("libcufft.so.11 could not be loaded");
    return SX_ERR_UNSUPPORTED;
  }
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0;
  SX_CUDA(cudaGetDevice(&dev));
  ZPlan *zp = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto &slot = g_plans[std::make_tuple(dev, nz, npts, plane_stride, sign)];
    if (!slot) {
      std::unique_ptr<ZPlan> np_(new ZPlan());
      SX_TRY(np_->spec.alloc((size_t)(nz / 2 + 1) * npts));
      int n[1] = {nz};
      int rembed[1] = {nz}, cembed[1] = {nz / 2 + 1};
      // real side: element stride = plane stride, transforms 1 apart;
      // complex side: [k][p], element stride npts, transforms 1 apart
      cufftResult r = sign == 1 ? api.planMany(&np_->plan, 1, n, rembed, plane_stride, 1, cembed, npts, 1,
                                               CUFFT_D2Z, npts)
                                : api.planMany(&np_->plan, 1, n, cembed, npts, 1, rembed, plane_stride, 1,
                                               CUFFT_Z2D, npts);
      if (r != CUFFT_SUCCESS) {
        set_error("cufftPlanMany(nz = %d, npts = %d): error %d", nz, npts, (int)r);
        return SX_ERR_CUDA;
      }
      slot = std::move(np_);
    }
    zp = slot.get();
  }
  // one transform at a time per plan (its workspace is shared)
  std::lock_guard<std::mutex> lk(g_mu);
  if (api.setStream(zp->plan, st) != CUFFT_SUCCESS) {
    set_error("cufftSetStream failed");
    return SX_ERR_CUDA;
  }
  const long long n = (long long)(nz / 2 + 1) * npts;
  const int grid = (int)std::min<long long>((n + 255) / 256, 8 * 148);
  if (sign == 1) {
    if (api.execD2Z(zp->plan, d_data, reinterpret_cast<cufftDoubleComplex *>(zp->spec.p)) != CUFFT_SUCCESS) {
      set_error("cufftExecD2Z failed");
      return SX_ERR_CUDA;
    }
    k_z_pack<<<grid, 256, 0, st>>>(zp->spec.p, d_data, nz, npts, plane_stride, 1.0 / nz);
  } else {
    k_z_unpack<<<grid, 256, 0, st>>>(d_data, zp->spec.p, nz, npts, plane_stride);
    if (api.execZ2D(zp->plan, reinterpret_cast<cufftDoubleComplex *>(zp->spec.p), d_data) != CUFFT_SUCCESS) {
      set_error("cufftExecZ2D failed");
      return SX_ERR_CUDA;
    }
  }
  SX_CUDA(cudaGetLastError());
  // the workspace is reused by the next call on this plan: finish here
  SX_CUDA(cudaStreamSynchronize(st));
  return SX_OK;
}
