// Masked multi-load PCG recurrences (exp/asg_gpu_resident_20261103/resident.py:39-58,119-131).
//
// Per iteration and active load l (alpha_l was formed by the operator's last block from p.q):
//   update_ur: u += alpha p; r -= alpha q; res2 = ||r||^2, sum r -> last block: iteration count,
//              keep / bad latches, new active mask, mean r (projection of the next Green input)
//   [Green passes: s.w and rz' = <v, G v> (= r.z), beta = rz'/rz]
//   update_p : p = (s.w - mean(s.w)) + beta p; thread 0 of block 0 also sets the CUDA-graph loop
//              condition (any load still active).
#include "pgj_internal.h"

namespace pgj {

template <typename T>
__global__ void __launch_bounds__(256) k_update_ur(int n, double* __restrict__ u64, T* __restrict__ uT, T* __restrict__ r,
                                                   const T* __restrict__ p, const T* __restrict__ q, LoadScalars* scal,
                                                   double* partials, int cap) {
  const size_t N = size_t(n) * n * n, N3 = 3 * N;
  const int load = blockIdx.y;
  LoadScalars& S = scal[load];
  if (!S.active) return;
  const double alpha = S.alpha;
  const T a = T(alpha);
  const size_t off = size_t(load) * N3;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  // grid-stride over nodes: 3 components per node so the component sums stay per-thread
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t k = off + 3 * i + c;
      const T pv = p[k];
      if (u64) u64[k] += alpha * double(pv);
      else uT[k] += a * pv;
      const T rv = r[k] - a * q[k];
      r[k] = rv;
      const double rd = double(rv);
      acc[0] += rd * rd;
      acc[1 + c] += rd;
    }
  }
  __shared__ double red[128];
  block_sum<4>(acc, red);
  double* part = partials + size_t(load) * kPartialQ * kMaxPartials;
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; ++k) part[k * kMaxPartials + blockIdx.x] = acc[k];
  if (!last_block(&S.ticket[kTicketUpdate], gridDim.x)) return;
  if (threadIdx.x < 32) {
    double v[4];
    for (int k = 0; k < 4; ++k) v[k] = warp_sum_partials(part + k * kMaxPartials, gridDim.x);
    if (threadIdx.x == 0) {
      const double res2 = v[0];
      const bool finite = isfinite(res2);
      const int it = S.iterations + 1;
      const bool valid = S.failed == 0;
      const bool keep = valid && finite && (res2 > S.target2) && (it < cap);
      S.iterations = it;
      S.bad = S.bad | (valid ? 0 : 1) | (finite ? 0 : 1);
      S.active = keep ? 1 : 0;
      S.res2 = res2;
      for (int c = 0; c < 3; ++c) S.mean_r[c] = v[1 + c] / double(N);
    }
  }
}

int launch_update_ur(pgj_ctx* c, int loads, int prec, double* u64, void* uT, cudaStream_t s) {
  dim3 grid(2 * 148, loads);
  if (prec == PGJ_FP32)
    k_update_ur<float><<<grid, 256, 0, s>>>(c->n, u64, static_cast<float*>(uT), static_cast<float*>(c->r),
                                            static_cast<const float*>(c->p), static_cast<const float*>(c->q), c->scal,
                                            c->partials, 4000);
  else
    k_update_ur<double><<<grid, 256, 0, s>>>(c->n, u64, static_cast<double*>(uT), static_cast<double*>(c->r),
                                             static_cast<const double*>(c->p), static_cast<const double*>(c->q),
                                             c->scal, c->partials, 4000);
  return check_launch();
}

// The loop body runs at most kMaxBodyRuns times per attempt whatever the masks say, so a graph
// WHILE loop can never spin unbounded (the per-load cap of 4000 iterations ends it first).
constexpr int kMaxBodyRuns = 4100;

template <typename T>
__global__ void __launch_bounds__(256) k_update_p(int n, int loads, T* __restrict__ p, const T* __restrict__ sw,
                                                  const LoadScalars* scal, int init, cudaGraphConditionalHandle h,
                                                  int set_cond, int* body_runs) {
  const size_t N3 = 3 * size_t(n) * n * n;
  const int load = blockIdx.y;
  if (set_cond && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
    int any = 0;
    for (int l = 0; l < loads; ++l) any |= scal[l].active;
    const int runs = ++body_runs[0];
    if (runs >= kMaxBodyRuns) body_runs[1] = 1;  // recorded: loop stopped by the bound
    cudaGraphSetConditional(h, (any && runs < kMaxBodyRuns) ? 1u : 0u);
  }
  const LoadScalars& S = scal[load];
  if (!S.active) return;
  const T m0 = T(S.mean_z[0]), m1 = T(S.mean_z[1]), m2 = T(S.mean_z[2]);
  const T beta = T(S.beta);
  const size_t off = size_t(load) * N3;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N3 / 3; i += size_t(gridDim.x) * blockDim.x) {
    const size_t k = off + 3 * i;
    const T z0 = sw[k] - m0, z1 = sw[k + 1] - m1, z2 = sw[k + 2] - m2;
    if (init) {
      p[k] = z0; p[k + 1] = z1; p[k + 2] = z2;
    } else {
      p[k] = z0 + beta * p[k];
      p[k + 1] = z1 + beta * p[k + 1];
      p[k + 2] = z2 + beta * p[k + 2];
    }
  }
}

int launch_update_p(pgj_ctx* c, int loads, int prec, bool init, cudaStream_t s, cudaGraphConditionalHandle h,
                    bool set_cond) {
  dim3 grid(2 * 148, loads);
  if (prec == PGJ_FP32)
    k_update_p<float><<<grid, 256, 0, s>>>(c->n, loads, static_cast<float*>(c->p), static_cast<const float*>(c->sw),
                                           c->scal, init ? 1 : 0, h, set_cond ? 1 : 0, c->cond);
  else
    k_update_p<double><<<grid, 256, 0, s>>>(c->n, loads, static_cast<double*>(c->p), static_cast<const double*>(c->sw),
                                            c->scal, init ? 1 : 0, h, set_cond ? 1 : 0, c->cond);
  return check_launch();
}

// active = ||r||^2 > target^2 and iterations < cap and not bad (resident.py:120); also resets the
// loop-body counter of the attempt.
__global__ void k_init_mask(int loads, LoadScalars* scal, int cap, int* body_runs) {
  const int l = threadIdx.x;
  if (l == 0) { body_runs[0] = 0; body_runs[1] = 0; }
  if (l >= loads) return;
  LoadScalars& S = scal[l];
  S.active = (S.res2 > S.target2) && (S.iterations < cap) && !S.bad ? 1 : 0;
  S.failed = 0;
}

int launch_init_mask(pgj_ctx* c, int loads, cudaStream_t s) {
  k_init_mask<<<1, 32, 0, s>>>(loads, c->scal, 4000, c->cond);
  return check_launch();
}

}  // namespace pgj
