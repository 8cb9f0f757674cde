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

// 48-byte chunks of a DOF vector: 6 doubles (2 nodes) or 12 floats (4 nodes), read as three
// 16-byte vectors; a chunk starts on a node, so element j of a chunk is component j % 3.
template <typename T> struct Chunk;
template <> struct Chunk<double> { static constexpr int CH = 6; using V = double2; };
template <> struct Chunk<float> { static constexpr int CH = 12; using V = float4; };

template <typename T>
__device__ __forceinline__ void load_chunk(const T* __restrict__ src, T (&v)[Chunk<T>::CH]) {
  using V = typename Chunk<T>::V;
  const V* s = reinterpret_cast<const V*>(src);
#pragma unroll
  for (int i = 0; i < 3; ++i) reinterpret_cast<V*>(v)[i] = s[i];
}
template <typename T>
__device__ __forceinline__ void store_chunk(T* __restrict__ dst, const T (&v)[Chunk<T>::CH]) {
  using V = typename Chunk<T>::V;
  V* d = reinterpret_cast<V*>(dst);
#pragma unroll
  for (int i = 0; i < 3; ++i) d[i] = reinterpret_cast<const V*>(v)[i];
}

// FLEX (FP32 flexible direction update): also r_new . z_prev, where z_prev = s.w - mean(s.w) of the
// previous Green apply, still held in `sw` (nothing writes it between update_p and this kernel).
template <typename T, typename U, bool FLEX = false>
__global__ void __launch_bounds__(256) k_update_ur(int n, U* __restrict__ u, T* __restrict__ r,
                                                   const T* __restrict__ p, const T* __restrict__ q, LoadScalars* scal,
                                                   double* partials, int cap, double rel_delta2,
                                                   const T* __restrict__ sw = nullptr) {
  constexpr int CH = Chunk<T>::CH;
  constexpr int NV = FLEX ? 5 : 4;
  const size_t N = size_t(n) * n * n, N3 = 3 * N;
  const int load = blockIdx.y;
  LoadScalars& S = scal[load];
  if (!S.active) return;
  const double alpha = S.alpha;
  const T a = T(alpha);
  const size_t off = size_t(load) * N3;
  double acc[NV] = {};
  const T mz[3] = {T(S.mean_z[0]), T(S.mean_z[1]), T(S.mean_z[2])};
  const size_t nch = N3 / CH;
  for (size_t ch = size_t(blockIdx.x) * blockDim.x + threadIdx.x; ch < nch; ch += size_t(gridDim.x) * blockDim.x) {
    const size_t k = off + ch * CH;
    T pv[CH], qv[CH], rv[CH];
    load_chunk<T>(p + k, pv);
    load_chunk<T>(q + k, qv);
    load_chunk<T>(r + k, rv);
    if constexpr (sizeof(U) == sizeof(T)) {
      U uv[CH];
      load_chunk<U>(u + k, uv);
#pragma unroll
      for (int j = 0; j < CH; ++j) uv[j] += U(alpha) * U(pv[j]);
      store_chunk<U>(u + k, uv);
    } else {
#pragma unroll
      for (int j = 0; j < CH; ++j) u[k + j] += alpha * double(pv[j]);
    }
#pragma unroll
    for (int j = 0; j < CH; ++j) {
      rv[j] = rv[j] - a * qv[j];
      const double rd = double(rv[j]);
      acc[0] += rd * rd;
      acc[1 + j % 3] += rd;
    }
    if constexpr (FLEX) {
      T zv[CH];
      load_chunk<T>(sw + k, zv);
#pragma unroll
      for (int j = 0; j < CH; ++j) acc[NV - 1] += double(rv[j]) * double(zv[j] - mz[j % 3]);
    }
    store_chunk<T>(r + k, rv);
  }
  __shared__ double red[32 * NV];
  block_sum<NV>(acc, red);
  double* part = partials + size_t(load) * kPartialQ * kMaxPartials;
  if (threadIdx.x == 0)
    for (int k = 0; k < NV; ++k) part[k * kMaxPartials + blockIdx.x] = acc[k];
  if (!last_block(&S.ticket[kTicketUpdate], gridDim.x)) return;
  if (threadIdx.x < 32) {
    double v[5] = {};
    for (int k = 0; k < NV; ++k) v[k] = warp_sum_partials(part + k * kMaxPartials, gridDim.x);
    if (threadIdx.x == 0) {
      if constexpr (FLEX) S.rz_cross = v[4];
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
      if (rel_delta2 > 0.0) {
        // reliable update: the recurrence residual fell by 1/delta since the last replacement, or the
        // recurrence believes it has converged; the FP64 true residual decides.
        const bool ok = valid && finite && it < cap;
        S.reliable = ok && ((keep && res2 < rel_delta2 * S.anchor) || (!keep && res2 <= S.target2)) ? 1 : 0;
      }
    }
  }
}

// Blocks per load for the vector updates: about four 48-byte chunks per thread (enough loads in
// flight per thread, few blocks paying the reduction), at least 16 and at most 296 per load.
static unsigned update_blocks(const pgj_ctx* c, int prec) {
  const size_t chunks = 3 * size_t(c->N) / (prec == PGJ_FP32 ? 12 : 6);
  size_t b = (chunks + 256 * 4 - 1) / (256 * 4);
  if (b < 16) b = 16;
  if (b > 296) b = 296;
  return unsigned(b);
}

int launch_update_ur(pgj_ctx* c, int loads, int prec, double* u64, void* uT, cudaStream_t s) {
  dim3 grid(update_blocks(c, prec), loads);
  const double rel = c->rel_delta2;
  if (prec == PGJ_FP32 && c->flex) {
    const float* sw = static_cast<const float*>(c->sw);
    if (u64)
      k_update_ur<float, double, true><<<grid, 256, 0, s>>>(c->n, u64, static_cast<float*>(c->r),
                                                            static_cast<const float*>(c->p),
                                                            static_cast<const float*>(c->q), c->scal, c->partials,
                                                            c->cap, rel, sw);
    else
      k_update_ur<float, float, true><<<grid, 256, 0, s>>>(c->n, static_cast<float*>(uT), static_cast<float*>(c->r),
                                                           static_cast<const float*>(c->p),
                                                           static_cast<const float*>(c->q), c->scal, c->partials,
                                                           c->cap, rel, sw);
  } else if (prec == PGJ_FP32) {
    if (u64)
      k_update_ur<float, double><<<grid, 256, 0, s>>>(c->n, u64, static_cast<float*>(c->r),
                                                      static_cast<const float*>(c->p), static_cast<const float*>(c->q),
                                                      c->scal, c->partials, c->cap, rel);
    else
      k_update_ur<float, float><<<grid, 256, 0, s>>>(c->n, static_cast<float*>(uT), static_cast<float*>(c->r),
                                                     static_cast<const float*>(c->p), static_cast<const float*>(c->q),
                                                     c->scal, c->partials, c->cap, rel);
  } else {
    k_update_ur<double, double><<<grid, 256, 0, s>>>(c->n, u64 ? u64 : static_cast<double*>(uT),
                                                     static_cast<double*>(c->r), static_cast<const double*>(c->p),
                                                     static_cast<const double*>(c->q), c->scal, c->partials, c->cap, rel);
  }
  return check_launch();
}

// The loop body runs at most `bound` (the iteration cap + 100) times per attempt whatever the masks
// say, so a graph WHILE loop can never spin unbounded (the per-load iteration cap ends it first).

template <typename T>
__global__ void __launch_bounds__(256) k_update_p(int n, int loads, T* __restrict__ p, const T* __restrict__ sw,
                                                  const LoadScalars* scal, int init, cudaGraphConditionalHandle h,
                                                  int set_cond, int* body_runs, int bound) {
  const size_t N3 = 3 * size_t(n) * n * n;
  const int load = blockIdx.y;
  if (set_cond && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
    int any = 0;
    for (int l = 0; l < loads; ++l) any |= scal[l].active;
    const int runs = ++body_runs[0];
    body_runs[5] += 1;                             // loop bodies over the whole solve (launch accounting)
    if (runs >= bound) body_runs[1] = 1;  // recorded: loop stopped by the bound
    cudaGraphSetConditional(h, (any && runs < bound) ? 1u : 0u);
  }
  const LoadScalars& S = scal[load];
  if (!S.active) return;
  constexpr int CH = Chunk<T>::CH;
  const T m[3] = {T(S.mean_z[0]), T(S.mean_z[1]), T(S.mean_z[2])};
  const T beta = T(S.beta);
  const size_t off = size_t(load) * N3;
  const size_t nch = N3 / CH;
  for (size_t ch = size_t(blockIdx.x) * blockDim.x + threadIdx.x; ch < nch; ch += size_t(gridDim.x) * blockDim.x) {
    const size_t k = off + ch * CH;
    T zv[CH], pv[CH];
    load_chunk<T>(sw + k, zv);
    if (init) {
#pragma unroll
      for (int j = 0; j < CH; ++j) pv[j] = zv[j] - m[j % 3];
    } else {
      load_chunk<T>(p + k, pv);
#pragma unroll
      for (int j = 0; j < CH; ++j) pv[j] = (zv[j] - m[j % 3]) + beta * pv[j];
    }
    store_chunk<T>(p + k, pv);
  }
}

int launch_update_p(pgj_ctx* c, int loads, int prec, bool init, cudaStream_t s, cudaGraphConditionalHandle h,
                    bool set_cond) {
  dim3 grid(update_blocks(c, prec), loads);
  if (prec == PGJ_FP32)
    k_update_p<float><<<grid, 256, 0, s>>>(c->n, loads, static_cast<float*>(c->p), static_cast<const float*>(c->sw),
                                           c->scal, init ? 1 : 0, h, set_cond ? 1 : 0, c->cond, c->cap + 100);
  else
    k_update_p<double><<<grid, 256, 0, s>>>(c->n, loads, static_cast<double*>(c->p), static_cast<const double*>(c->sw),
                                            c->scal, init ? 1 : 0, h, set_cond ? 1 : 0, c->cond, c->cap + 100);
  return check_launch();
}

// active = ||r||^2 > target^2 and iterations < cap and not bad (resident.py:120); also resets the
// loop-body counter of the attempt. Loads of a design that took its last attempt stay inactive.
__global__ void k_init_mask(int loads, LoadScalars* scal, int cap, int* body_runs) {
  if (threadIdx.x == 0) body_runs[0] = 0;
  for (int l = threadIdx.x; l < loads; l += blockDim.x) {
    LoadScalars& S = scal[l];
    S.active = (S.res2 > S.target2) && (S.iterations < cap) && !S.bad && !S.frozen ? 1 : 0;
    S.failed = 0;
  }
}

int launch_init_mask(pgj_ctx* c, int loads, cudaStream_t s) {
  k_init_mask<<<1, 32, 0, s>>>(loads, c->scal, c->cap, c->cond);
  return check_launch();
}

// ------------------------------------------------------------------------------ mixed refinement
// Start of one refinement sweep, per load: the FP64 certificate decides whether the load still needs
// a correction; r_in = T(r64), d = 0; the inner target is inner_rtol * ||r64||.
// `planar`: the FP32 vectors r and d are component-planar, (3, N) per load (slab-fused contexts);
// the FP64 vectors are node-major interleaved either way.
__device__ __forceinline__ size_t pidx(size_t node, int c, size_t N, int planar) {
  return planar ? size_t(c) * N + node : 3 * node + c;
}

template <typename T>
__global__ void __launch_bounds__(256) k_inner_start(int n, const double* __restrict__ r64, T* __restrict__ r,
                                                     T* __restrict__ d, const LoadScalars* out_scal,
                                                     LoadScalars* in_scal, double* partials, double inner_rtol,
                                                     int* body_runs, int planar) {
  const size_t N = size_t(n) * n * n, N3 = 3 * N;
  const int load = blockIdx.y;
  const LoadScalars& O = out_scal[load];
  LoadScalars& S = in_scal[load];
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) body_runs[0] = 0;
  const bool done = isfinite(O.absolute) && O.absolute * O.absolute <= O.target2 && !O.bad;
  if (done) {
    if (blockIdx.x == 0 && threadIdx.x == 0) { S.active = 0; S.touched = 0; S.iterations = 0; }
    return;
  }
  const size_t off = size_t(load) * N3;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t k = off + 3 * i + c, kt = off + pidx(i, c, N, planar);
      const T v = T(r64[k]);
      r[kt] = v;
      d[kt] = T(0);
      const double dv = double(v);
      acc[0] += dv * dv;
      acc[1 + c] += dv;
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
      const double t = inner_rtol * O.absolute;
      S.target2 = t * t;
      S.res2 = v[0];
      for (int c = 0; c < 3; ++c) S.mean_r[c] = v[1 + c] / double(N);
      S.iterations = 0;
      S.bad = 0;
      S.failed = 0;
      S.touched = 1;
      S.active = (v[0] > S.target2) && isfinite(v[0]) ? 1 : 0;
    }
  }
}

// End of a sweep: x += d for touched loads; iteration and latch bookkeeping on the outer record.
template <typename T>
__global__ void __launch_bounds__(256) k_inner_finish(int n, double* __restrict__ x, const T* __restrict__ d,
                                                      LoadScalars* out_scal, const LoadScalars* in_scal, int planar) {
  const size_t N = size_t(n) * n * n, N3 = 3 * N;
  const int load = blockIdx.y;
  const LoadScalars& S = in_scal[load];
  if (!S.touched) return;
  const size_t off = size_t(load) * N3;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x)
#pragma unroll
    for (int c = 0; c < 3; ++c) x[off + 3 * i + c] += double(d[off + pidx(i, c, N, planar)]);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    out_scal[load].total_iterations += S.iterations;
    out_scal[load].bad |= S.bad;
  }
}

int launch_inner_start(pgj_ctx* c, int loads, double inner_rtol, cudaStream_t s) {
  dim3 grid(2 * 148, loads);
  k_inner_start<float><<<grid, 256, 0, s>>>(c->n, c->r64, static_cast<float*>(c->r), static_cast<float*>(c->d),
                                            c->scal_out, c->scal_in, c->partials, inner_rtol, c->cond, c->fused);
  return check_launch();
}

int launch_inner_finish(pgj_ctx* c, int loads, cudaStream_t s) {
  dim3 grid(2 * 148, loads);
  k_inner_finish<float><<<grid, 256, 0, s>>>(c->n, c->x, static_cast<const float*>(c->d), c->scal_out, c->scal_in,
                                             c->fused);
  return check_launch();
}

// ------------------------------------------------------------------------------ reliable updates
// Mixed solve: one FP32 CG recurrence per load; at chosen iterations the FP32 correction d is folded
// into the FP64 solution x and the recurrence residual is replaced by the FP64 true residual f - K x.

// r_in = T(r64), d = 0, recurrence scalars from the FP64 certificate (attempt start)
template <typename T>
__global__ void __launch_bounds__(256) k_rel_start(int n, const double* __restrict__ r64, T* __restrict__ r,
                                                   T* __restrict__ d, const LoadScalars* out, LoadScalars* in, int cap,
                                                   int* body_runs, int planar) {
  const size_t N = size_t(n) * n * n, N3 = 3 * N;
  const int load = blockIdx.y;
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) body_runs[0] = 0;
  const size_t off = size_t(load) * N3;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t kt = off + pidx(i, c, N, planar);
      r[kt] = T(r64[off + 3 * i + c]);
      d[kt] = T(0);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const LoadScalars& O = out[load];
    LoadScalars& S = in[load];
    S.res2 = O.res2;
    S.anchor = O.res2;
    S.target2 = O.target2;
    for (int c = 0; c < 3; ++c) S.mean_r[c] = O.mean_r[c];
    S.iterations = O.iterations;
    S.bad = O.bad;
    S.failed = 0;
    S.reliable = 0;
    S.active = (O.res2 > O.target2) && (O.iterations < cap) && !O.bad && !O.frozen ? 1 : 0;
  }
}

// IF-node condition: any load flagged for a true-residual replacement
__global__ void k_rel_cond(int loads, const LoadScalars* in, cudaGraphConditionalHandle h, int* counters) {
  if (threadIdx.x != 0) return;
  int any = 0;
  for (int l = 0; l < loads; ++l) any |= in[l].reliable;
  if (any) counters[3] += 1;  // replacements taken (launch accounting)
  cudaGraphSetConditional(h, any ? 1u : 0u);
}

// x += d, d = 0 for flagged loads (all loads when `all`)
template <typename T>
__global__ void __launch_bounds__(256) k_rel_fold(int n, double* __restrict__ x, T* __restrict__ d,
                                                  const LoadScalars* in, LoadScalars* out, int all, int planar) {
  const size_t N = size_t(n) * n * n, N3 = 3 * N;
  const int load = blockIdx.y;
  if (!all && !in[load].reliable) return;
  if (all && blockIdx.x == 0 && threadIdx.x == 0) {
    // end of the attempt: the recurrence's bookkeeping becomes the certificate's
    out[load].iterations = in[load].iterations;
    out[load].bad |= in[load].bad;
  }
  const size_t off = size_t(load) * N3;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t kt = off + pidx(i, c, N, planar);
      x[off + 3 * i + c] += double(d[kt]);
      d[kt] = T(0);
    }
  }
}

// flagged loads: r_in = T(r64) (the true residual the FP64 operator just produced); the last block
// resets the recurrence scalars to it and decides whether the load keeps iterating
template <typename T>
__global__ void __launch_bounds__(256) k_rel_sync(int n, const double* __restrict__ r64, T* __restrict__ r,
                                                  const LoadScalars* out, LoadScalars* in, int cap, int planar) {
  const size_t N = size_t(n) * n * n, N3 = 3 * N;
  const int load = blockIdx.y;
  LoadScalars& S = in[load];
  if (!S.reliable) return;
  const size_t off = size_t(load) * N3;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x)
#pragma unroll
    for (int c = 0; c < 3; ++c) r[off + pidx(i, c, N, planar)] = T(r64[off + 3 * i + c]);
  if (!last_block(&S.ticket[kTicketAux2], gridDim.x)) return;
  if (threadIdx.x == 0) {
    const LoadScalars& O = out[load];
    S.res2 = O.res2;
    S.anchor = O.res2;
    for (int c = 0; c < 3; ++c) S.mean_r[c] = O.mean_r[c];
    S.active = isfinite(O.res2) && O.res2 > S.target2 && S.iterations < cap && !S.bad ? 1 : 0;
    S.reliable = 0;
  }
}

// Device-side restart decision after an attempt's certification (resident.py:202-205), per design
// (the loads [g lpd, (g+1) lpd) of a batched context; a plain context is one design): another
// attempt only when some certificate of the design failed, fewer than two restarts were taken, none
// of its loads latched `bad`, no failing load reached the iteration cap and the loop bound was not
// hit. A design that stops is frozen: later attempts of its batch-mates leave its loads untouched.
__global__ void k_decide(int loads, int lpd, LoadScalars* out, int* counters, cudaGraphConditionalHandle h,
                         int cap) {
  if (threadIdx.x != 0) return;
  bool any_again = false;
  for (int g = 0; g * lpd < loads; ++g) {
    bool all = true, anybad = false, capped = false;
    const int l1 = min(loads, (g + 1) * lpd);
    if (out[g * lpd].frozen) continue;
    for (int l = g * lpd; l < l1; ++l) {
      const LoadScalars& S = out[l];
      const bool ok = isfinite(S.absolute) && S.absolute * S.absolute <= S.target2 && !S.bad;
      all = all && ok;
      anybad = anybad || S.bad;
      capped = capped || (!ok && S.iterations >= cap);
    }
    const bool again = !all && out[g * lpd].restarts < 2 && !anybad && !capped && !counters[1] && !counters[2];
    for (int l = g * lpd; l < l1; ++l) {
      if (again) out[l].restarts += 1;
      else out[l].frozen = 1;
    }
    any_again = any_again || again;
  }
  if (any_again) counters[4] += 1;  // attempts after the first, over the whole context
  cudaGraphSetConditional(h, any_again ? 1u : 0u);
}

int launch_decide(pgj_ctx* c, int loads, cudaGraphConditionalHandle h, cudaStream_t s) {
  k_decide<<<1, 32, 0, s>>>(loads, c->lpd, c->scal_out, c->cond, h, c->cap);
  return check_launch();
}

int launch_rel_start(pgj_ctx* c, int loads, cudaStream_t s) {
  k_rel_start<float><<<dim3(2 * 148, loads), 256, 0, s>>>(c->n, c->r64, static_cast<float*>(c->r),
                                                          static_cast<float*>(c->d), c->scal_out, c->scal_in, c->cap,
                                                          c->cond, c->fused);
  return check_launch();
}
int launch_rel_cond(pgj_ctx* c, int loads, cudaGraphConditionalHandle h, cudaStream_t s) {
  k_rel_cond<<<1, 32, 0, s>>>(loads, c->scal_in, h, c->cond);
  return check_launch();
}
int launch_rel_fold(pgj_ctx* c, int loads, bool all, cudaStream_t s) {
  k_rel_fold<float><<<dim3(2 * 148, loads), 256, 0, s>>>(c->n, c->x, static_cast<float*>(c->d), c->scal_in,
                                                         c->scal_out, all ? 1 : 0, c->fused);
  return check_launch();
}
int launch_rel_sync(pgj_ctx* c, int loads, cudaStream_t s) {
  k_rel_sync<float><<<dim3(2 * 148, loads), 256, 0, s>>>(c->n, c->r64, static_cast<float*>(c->r), c->scal_out,
                                                         c->scal_in, c->cap, c->fused);
  return check_launch();
}

}  // namespace pgj
