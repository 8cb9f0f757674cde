// Design-update chains kept on the device: density filters, projection + SIMP, and the optimality
// criteria (OC) volume bisection.
//
// Study II (paper conventions, exp/asg_sctop_reproduction_20261105/outer.cu:8-39 and
// reproduction.py:69-118): clipped cone filter, tanh(beta, eta) projection, damped OC
// x' = clip(x max(1e-10, ratio/mid)^exponent, max(floor, x-move), min(1, x+move)), MATLAB
// bisection stop (hi-lo)/(hi+lo) <= 1e-4, at most 180 steps.
// Study I (exp/asg_gpu_resident_20261103/outer.cu:7-37, outer.py:26-44): periodic separable
// Gaussian (scipy.ndimage correlation order), tanh projection at 1/2, SIMP eta=1e-4, 45 steps.
//
// The bisection state lives in a 4-double device record {lo, hi, flag, steps}; every step's
// kernels return immediately once the flag is cleared, so the whole chain is issued without any
// host synchronisation and reads back only at the end.
#include "pgj_internal.h"
#include <cmath>
#include <vector>

namespace pgj {

// Clipped cone filter y(p) = sum_j w_j x(p + d_j) over the taps whose neighbour lies inside the grid
// (no periodic wrap). A block covers 32 x 8 columns of the (x, y) plane (x fastest, one warp per
// row) in one z plane (and every gridDim.z-th plane after it); the tap table is staged in shared
// memory (dx, dy, dz, the neighbour's linear offset and the weight), kConeChunk taps at a time, so
// every thread reads a tap as a broadcast. Taps are summed in table order with one fused
// multiply-add each, the order of the reference's loop, so the result does not depend on the
// tiling. `flag` (the OC bisection record) ends the launch once the bisection has stopped.
constexpr int kConeChunk = 512;
constexpr int kConeX = 32, kConeY = 8;
struct ConeTap {
  int dx, dy, dz, pad;
  long long lin;  // (dz n + dy) n + dx
  double w;
};

__global__ void __launch_bounds__(kConeX * kConeY) k_cone_filter(int n, const int32_t* __restrict__ offsets,
                                                                 const double* __restrict__ weights, int count,
                                                                 const double* __restrict__ x,
                                                                 double* __restrict__ y, const double* flag) {
  if (flag && flag[2] == 0.0) return;
  __shared__ ConeTap taps[kConeChunk];
  const int tid = threadIdx.y * kConeX + threadIdx.x;
  const int cx = blockIdx.x * kConeX + threadIdx.x, cy = blockIdx.y * kConeY + threadIdx.y;
  const bool inside = cx < n && cy < n;
  const unsigned un = unsigned(n);
  auto stage = [&](int first, int m) {
    for (int j = tid; j < m; j += kConeX * kConeY) {
      ConeTap t;
      t.dx = offsets[3 * (first + j)];
      t.dy = offsets[3 * (first + j) + 1];
      t.dz = offsets[3 * (first + j) + 2];
      t.pad = 0;
      t.lin = (static_cast<long long>(t.dz) * n + t.dy) * n + t.dx;
      t.w = weights[first + j];
      taps[j] = t;
    }
  };
  const bool resident = count <= kConeChunk;  // the whole table stays staged across the z planes
  if (resident) stage(0, count);
  __syncthreads();
  for (int cz = blockIdx.z; cz < n; cz += gridDim.z) {
    const size_t at = (size_t(cz) * n + cy) * n + cx;
    double sum = 0.0;
    for (int first = 0; first < count; first += kConeChunk) {
      const int m = min(kConeChunk, count - first);
      if (!resident) {
        __syncthreads();  // the previous chunk has been read by every thread
        stage(first, m);
        __syncthreads();
      }
      if (!inside) continue;
      for (int j = 0; j < m; ++j) {
        const ConeTap& t = taps[j];
        if (unsigned(cx + t.dx) < un && unsigned(cy + t.dy) < un && unsigned(cz + t.dz) < un)
          sum += t.w * x[static_cast<long long>(at) + t.lin];
      }
    }
    if (inside) y[at] = sum;
  }
}

__device__ __forceinline__ void paper_phys(double t, double hs, double beta, double eta, double emin, double& ph,
                                           double& dp, double& a) {
  const double den = tanh(beta * eta) + tanh(beta * (1 - eta));
  const double q = tanh(beta * (t / hs - eta));
  const double rho = (tanh(beta * eta) + q) / den;
  ph = rho;
  dp = beta * (1 - q * q) / den;
  a = emin + (1 - emin) * rho * rho * rho;
}

__global__ void k_paper_project(size_t N, const double* __restrict__ t, const double* __restrict__ hs, double beta,
                                double eta, double emin, double* __restrict__ ph, double* __restrict__ dp,
                                double* __restrict__ a) {
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
    double p, d, aa;
    paper_phys(t[i], hs[i], beta, eta, emin, p, d, aa);
    ph[i] = p; dp[i] = d; a[i] = aa;
  }
}

// g = dp (3 (1-emin) ph^2) energy / hs ; v = dp / hs (filter inputs of the OC sensitivities)
__global__ void k_paper_sens_in(size_t N, const double* __restrict__ ph, const double* __restrict__ dp,
                                const double* __restrict__ hs, const double* __restrict__ energy, double emin,
                                double* __restrict__ gin, double* __restrict__ vin) {
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
    gin[i] = dp[i] * (3 * (1 - emin) * (ph[i] * ph[i])) * energy[i] / hs[i];
    vin[i] = dp[i] / hs[i];
  }
}

// ratio = -(g / N) / dv, stored in place of g (reproduction.py:92-95)
__global__ void k_paper_ratio(size_t N, double* __restrict__ g, const double* __restrict__ dv, double* bounds) {
  const double dN = double(N);
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x)
    g[i] = -(g[i] / dN) / dv[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) { bounds[0] = 0.0; bounds[1] = 1e9; bounds[2] = 1.0; bounds[3] = 0.0; }
}

__global__ void k_paper_candidate(size_t N, const double* __restrict__ x, const double* __restrict__ ratio,
                                  const double* bounds, double move, double exponent, double floor_,
                                  double* __restrict__ y) {
  if (bounds[2] == 0.0) return;
  const double mid = 0.5 * (bounds[0] + bounds[1]);
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
    const double v = x[i] * pow(fmax(1e-10, ratio[i] / mid), exponent);
    y[i] = fmax(floor_, fmax(x[i] - move, fmin(1.0, fmin(x[i] + move, v))));
  }
}

// trial projection, volume mean and the bisection update in the last block
__global__ void k_paper_volume(size_t N, const double* __restrict__ t, const double* __restrict__ hs, double beta,
                               double eta, double emin, double target, double* bounds, double* partials,
                               int* ticket) {
  if (bounds[2] == 0.0) return;
  double acc[1] = {0.0};
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
    double p, d, a;
    paper_phys(t[i], hs[i], beta, eta, emin, p, d, a);
    acc[0] += p;
  }
  __shared__ double red[32];
  block_sum<1>(acc, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc[0];
  if (!last_block(ticket, gridDim.x)) return;
  if (threadIdx.x < 32) {
    const double s = warp_sum_partials(partials, gridDim.x);
    if (threadIdx.x == 0) {
      const double vol = s / double(N);
      const double mid = 0.5 * (bounds[0] + bounds[1]);
      if (vol > target) bounds[0] = mid; else bounds[1] = mid;
      bounds[3] += 1.0;
      bounds[2] = ((bounds[1] - bounds[0]) / (bounds[1] + bounds[0]) > 1e-4 && bounds[1] > 1e-40) ? 1.0 : 0.0;
    }
  }
}

// max |xnew - x| (single block reduction into out[0])
__global__ void k_absmax_diff(size_t N, const double* __restrict__ a, const double* __restrict__ b, double* out) {
  double m = 0.0;
  for (size_t i = threadIdx.x; i < N; i += blockDim.x) m = fmax(m, fabs(a[i] - b[i]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) out[0] = m;
  }
}

// --------------------------------------------------------------------------- Study I
// y[i] = w[r] x[i] + sum_k w[r+k] (x[i-k] + x[i+k]) along one periodic axis.
__global__ void k_gauss_axis(int n, int axis, const double* __restrict__ w, int radius, const double* __restrict__ x,
                             double* __restrict__ y) {
  const size_t N = size_t(n) * n * n;
  const size_t stride = axis == 0 ? size_t(n) * n : (axis == 1 ? size_t(n) : 1);
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
    const int coord = int((i / stride) % n);
    double v = w[radius] * x[i];
    for (int k = 1; k <= radius; ++k) {
      int lo = (coord - k) % n;
      if (lo < 0) lo += n;
      const int hi = (coord + k) % n;
      v += w[radius + k] * (x[i + (long long)(lo - coord) * (long long)stride] + x[i + (long long)(hi - coord) * (long long)stride]);
    }
    y[i] = v;
  }
}

__device__ __forceinline__ void s1_phys(double t, double b, double& p, double& d, double& a) {
  const double half = tanh(0.5 * b), q = tanh(b * (t - 0.5));
  p = (half + q) / (2 * half);
  d = b * (1 - q * q) / (2 * half);
  a = 1e-4 + (1.0 - 1e-4) * p * p * p;
}

__global__ void k_s1_project(size_t N, const double* __restrict__ t, double beta, double* __restrict__ ph,
                             double* __restrict__ dp, double* __restrict__ a) {
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
    double p, d, aa;
    s1_phys(t[i], beta, p, d, aa);
    ph[i] = p; dp[i] = d; a[i] = aa;
  }
}

__global__ void k_s1_sens_in(size_t N, const double* __restrict__ ph, const double* __restrict__ dp,
                             const double* __restrict__ energy, double* __restrict__ gin) {
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x)
    gin[i] = dp[i] * 3 * (1. - 1e-4) * (ph[i] * ph[i]) * energy[i];
}

// ratio = max(g,1e-30)/max(dv,1e-30) in place; hi bound = max(ratio) * 1e4 (single-block max)
__global__ void k_s1_ratio(size_t N, double* __restrict__ g, const double* __restrict__ dv, double* bounds) {
  double m = 0.0;
  for (size_t i = threadIdx.x; i < N; i += blockDim.x) {
    const double r = fmax(g[i], 1e-30) / fmax(dv[i], 1e-30);
    g[i] = r;
    m = fmax(m, r);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) { bounds[0] = 0.0; bounds[1] = m * 1e4; bounds[2] = 1.0; bounds[3] = 0.0; }
  }
}

__global__ void k_s1_candidate(size_t N, const double* __restrict__ x, const double* __restrict__ ratio,
                               const double* bounds, double move, double* __restrict__ y) {
  const double lam = fmax((bounds[0] + bounds[1]) * 0.5, 1e-30);
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
    const double lo = fmax(0., x[i] - move), hi = fmin(1., x[i] + move);
    y[i] = fmin(hi, fmax(lo, x[i] * sqrt(ratio[i] / lam)));
  }
}

__global__ void k_s1_volume(size_t N, const double* __restrict__ t, double beta, double target, double* bounds,
                            double* partials, int* ticket) {
  double acc[1] = {0.0};
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
    double p, d, a;
    s1_phys(t[i], beta, p, d, a);
    acc[0] += p;
  }
  __shared__ double red[32];
  block_sum<1>(acc, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc[0];
  if (!last_block(ticket, gridDim.x)) return;
  if (threadIdx.x < 32) {
    const double s = warp_sum_partials(partials, gridDim.x);
    if (threadIdx.x == 0) {
      const double mid = (bounds[0] + bounds[1]) * 0.5;
      if (s / double(N) > target) bounds[0] = mid; else bounds[1] = mid;
      bounds[3] += 1.0;
    }
  }
}

}  // namespace pgj

using namespace pgj;

namespace {
constexpr int kOCBlocks = 296;
// cone filter launch: one block per 32 x 8 column tile and z plane (n = 64: 1024 blocks, up to
// seven resident per SM). Splitting the planes over about kOCBlocks blocks, each walking three or
// four of them, measured 61.5 against 34.8 us at n = 64 (93 taps)
dim3 cone_grid(int n) {
  const int bx = (n + kConeX - 1) / kConeX, by = (n + kConeY - 1) / kConeY;
  const int bz = std::min(n, 65535);  // the kernel walks the planes beyond the grid's z limit
  return dim3(unsigned(bx), unsigned(by), unsigned(bz));
}
const dim3 kConeBlock(kConeX, kConeY);
// scratch layout for the OC chains: 4 fields of N doubles, then 8 doubles of bisection state,
// an int ticket and kOCBlocks partials.
struct OCScratch {
  double *f0, *f1, *f2, *f3, *bounds, *partials;
  int* ticket;
};
OCScratch oc_scratch(double* scratch, size_t N) {
  OCScratch s;
  s.f0 = scratch; s.f1 = scratch + N; s.f2 = scratch + 2 * N; s.f3 = scratch + 3 * N;
  s.bounds = scratch + 4 * N;
  s.ticket = reinterpret_cast<int*>(s.bounds + 8);
  s.partials = s.bounds + 16;
  return s;
}
}  // namespace

extern "C" {

int pgj_cone_filter(int n, const int32_t* offsets, const double* weights, int count, const double* x, double* y,
                    void* stream) {
  if (n < 2 || !offsets || !weights || count < 1 || !x || !y) return PGJ_ERR_ARGUMENT;
  k_cone_filter<<<cone_grid(n), kConeBlock, 0, static_cast<cudaStream_t>(stream)>>>(n, offsets, weights, count, x, y,
                                                                                   nullptr);
  return check_launch();
}

int pgj_paper_project(int n, const double* t, const double* hs, double beta, double eta, double emin, double* ph,
                      double* dp, double* a, void* stream) {
  if (n < 2 || !t || !hs || !ph || !dp || !a) return PGJ_ERR_ARGUMENT;
  k_paper_project<<<kOCBlocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(size_t(n) * n * n, t, hs, beta, eta, emin,
                                                                            ph, dp, a);
  return check_launch();
}

// scratch: 4 N + 16 + kOCBlocks doubles (see pgj.h: "4 n^3 float64" plus a small tail; callers
// allocate 4 n^3 + 512 doubles).
int pgj_paper_oc(int n, const int32_t* offsets, const double* weights, int count, const double* x, const double* ph,
                 const double* dp, const double* hs, const double* energy, double volume, double beta, double eta,
                 double emin, double move, double exponent, double floor_, double* xnew, double* scratch, int* steps,
                 double* change, void* stream) {
  if (n < 2 || !offsets || !weights || count < 1 || !x || !ph || !dp || !hs || !energy || !xnew || !scratch)
    return PGJ_ERR_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t N = size_t(n) * n * n;
  OCScratch w = oc_scratch(scratch, N);
  cudaError_t e = cudaMemsetAsync(w.ticket, 0, sizeof(int), s);
  if (e != cudaSuccess) return set_cuda_error(e);
  // g -> f0 (then ratio), dv -> f1
  k_paper_sens_in<<<kOCBlocks, 256, 0, s>>>(N, ph, dp, hs, energy, emin, w.f2, w.f3);
  k_cone_filter<<<cone_grid(n), kConeBlock, 0, s>>>(n, offsets, weights, count, w.f2, w.f0, nullptr);
  k_cone_filter<<<cone_grid(n), kConeBlock, 0, s>>>(n, offsets, weights, count, w.f3, w.f1, nullptr);
  k_paper_ratio<<<kOCBlocks, 256, 0, s>>>(N, w.f0, w.f1, w.bounds);
  int st = check_launch();
  if (st) return st;
  for (int it = 0; it < 180; ++it) {
    k_paper_candidate<<<kOCBlocks, 256, 0, s>>>(N, x, w.f0, w.bounds, move, exponent, floor_, xnew);
    k_cone_filter<<<cone_grid(n), kConeBlock, 0, s>>>(n, offsets, weights, count, xnew, w.f2, w.bounds);
    k_paper_volume<<<kOCBlocks, 256, 0, s>>>(N, w.f2, hs, beta, eta, emin, volume, w.bounds, w.partials, w.ticket);
  }
  k_absmax_diff<<<1, 1024, 0, s>>>(N, xnew, x, w.bounds + 4);
  if ((st = check_launch())) return st;
  if (!steps && !change) return PGJ_OK;  // enqueue only: the record stays in scratch[4N + 3 .. 4N + 4]
  double host[8];
  e = cudaMemcpyAsync(host, w.bounds, sizeof(host), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return set_cuda_error(e);
  if (steps) *steps = int(host[3]);
  if (change) *change = host[4];
  return PGJ_OK;
}

int pgj_gaussian_filter(int n, const double* weights, int radius, const double* x, double* y, double* scratch,
                        void* stream) {
  if (n < 2 || !weights || radius < 0 || 2 * radius + 1 > 4 * n + 1 || !x || !y || !scratch) return PGJ_ERR_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_gauss_axis<<<kOCBlocks, 256, 0, s>>>(n, 0, weights, radius, x, scratch);
  k_gauss_axis<<<kOCBlocks, 256, 0, s>>>(n, 1, weights, radius, scratch, scratch + size_t(n) * n * n);
  k_gauss_axis<<<kOCBlocks, 256, 0, s>>>(n, 2, weights, radius, scratch + size_t(n) * n * n, y);
  return check_launch();
}

int pgj_study1_project(int n, const double* t, double beta, double* ph, double* dp, double* a, void* stream) {
  if (n < 2 || !t || !ph || !dp || !a) return PGJ_ERR_ARGUMENT;
  k_s1_project<<<kOCBlocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(size_t(n) * n * n, t, beta, ph, dp, a);
  return check_launch();
}

int pgj_study1_oc(int n, const double* weights, int radius, const double* x, const double* ph, const double* dp,
                  const double* energy, double beta, double volume, double move, double* xnew, double* scratch,
                  double* change, void* stream) {
  if (n < 2 || !weights || !x || !ph || !dp || !energy || !xnew || !scratch) return PGJ_ERR_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t N = size_t(n) * n * n;
  // fields: f0 ratio, f1 dv, f2/f3 filter temporaries; gaussian scratch reuses f2|f3 (2N)
  OCScratch w = oc_scratch(scratch, N);
  cudaError_t e = cudaMemsetAsync(w.ticket, 0, sizeof(int), s);
  if (e != cudaSuccess) return set_cuda_error(e);
  k_s1_sens_in<<<kOCBlocks, 256, 0, s>>>(N, ph, dp, energy, xnew);
  int st;
  if ((st = pgj_gaussian_filter(n, weights, radius, xnew, w.f0, w.f2, stream))) return st;
  if ((st = pgj_gaussian_filter(n, weights, radius, dp, w.f1, w.f2, stream))) return st;
  k_s1_ratio<<<1, 1024, 0, s>>>(N, w.f0, w.f1, w.bounds);
  for (int it = 0; it < 45; ++it) {
    k_s1_candidate<<<kOCBlocks, 256, 0, s>>>(N, x, w.f0, w.bounds, move, xnew);
    if ((st = pgj_gaussian_filter(n, weights, radius, xnew, w.f1, w.f2, stream))) return st;
    k_s1_volume<<<kOCBlocks, 256, 0, s>>>(N, w.f1, beta, volume, w.bounds, w.partials, w.ticket);
  }
  // the candidate of the last bisection is the returned design (study.py:91-100)
  k_absmax_diff<<<1, 1024, 0, s>>>(N, xnew, x, w.bounds + 4);
  if ((st = check_launch())) return st;
  if (!change) return PGJ_OK;  // enqueue only: the change stays in scratch[4N + 4]
  double host[8];
  e = cudaMemcpyAsync(host, w.bounds, sizeof(host), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return set_cuda_error(e);
  if (change) *change = host[4];
  return PGJ_OK;
}

}  // extern "C"
