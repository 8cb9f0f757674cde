// Shared definitions for the libpgj kernels (sm_100a).
//
// Layouts (all device memory, owned by the caller):
//   DOF vector    : (L, N, 3) node-major, xyz interleaved, nodes in (z, y, x) order, N = n^3.
//   scalar field  : (N,) in (z, y, x) order (density multiplier a, sensitivities, ...).
//   half spectrum : (L, 3, n, n, ns) complex, ns = n/2 + 1, component-planar, kx fastest.
//   symbol        : (6, n, n, ns) real; xx, yy, zz, xy, xz, yz with 1/N folded in.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "../../include/pgj.h"

namespace pgj {

constexpr int kMaxLoads = 8;          // right-hand sides per design
constexpr int kMaxDesigns = 16;       // designs of one batched context
constexpr int kMaxTotalLoads = kMaxLoads * kMaxDesigns;
constexpr int kMaxStages = 8;

__host__ __device__ __forceinline__ int wrapi(int x, int n) { return x < 0 ? x + n : (x >= n ? x - n : x); }

// --------------------------------------------------------------------------- TMA bulk copies
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// --- TMA (bulk async copy) staging: one elected thread copies whole rows into shared memory and
// the block waits on an mbarrier whose transaction count is the plane's byte size.
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tma_row(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after kMaxTries polls (each poll may suspend briefly in hardware).
constexpr int kMaxTries = 1 << 20;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int max_tries = kMaxTries) {
  for (int i = 0; i < max_tries; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Bulk store shared -> global (the async proxy reads shared memory; make generic writes visible first
// with fence_proxy_async() and a block barrier, and wait for the reads before the buffer is reused
// or the block exits).
__device__ __forceinline__ void tma_store_row(void* gdst, const void* ssrc, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(gdst), "r"(smem_u32(ssrc)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void tma_store_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void tma_store_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void tma_store_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }

// --------------------------------------------------------------------------- fast division
// Quotient of a non-negative int below 2^31 by a fixed divisor d with one multiply-high and a
// shift: m = ceil(2^p / d), p = 31 + ceil(log2 d) (the divisor-reciprocal method; checked
// exhaustively on the host for the divisors used here).
struct FastDiv {
  unsigned d, m, s;
};
inline FastDiv make_fastdiv(unsigned d) {
  FastDiv f;
  f.d = d;
  if (d <= 1) { f.m = 0; f.s = 0; return f; }
  unsigned l = 0;
  while ((1u << l) < d) ++l;
  const unsigned p = 31 + l;
  f.m = unsigned(((1ull << p) + d - 1) / d);
  f.s = p - 32;
  return f;
}
__device__ __forceinline__ int fdiv(int x, const FastDiv& f) {
  return f.d <= 1 ? x : int(__umulhi(unsigned(x), f.m) >> f.s);
}

// --------------------------------------------------------------------------- complex
template <typename T> struct Cx;
template <> struct Cx<double> { using type = double2; };
template <> struct Cx<float> { using type = float2; };
template <typename T> using cplx = typename Cx<T>::type;

template <typename C> __device__ __forceinline__ C cmk(double re, double im) { C c; c.x = re; c.y = im; return c; }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { C c; c.x = a.x + b.x; c.y = a.y + b.y; return c; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { C c; c.x = a.x - b.x; c.y = a.y - b.y; return c; }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C c; c.x = a.x * b.x - a.y * b.y; c.y = a.x * b.y + a.y * b.x; return c;
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
  C c; c.x = a.x * b.x + a.y * b.y; c.y = a.y * b.x - a.x * b.y; return c;
}
template <typename C> __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
// FP32 complex arithmetic as packed FP32 operations (two results per instruction on sm_100);
// adds and subtracts round exactly like their scalar forms
template <> __device__ __forceinline__ float2 cadd<float2>(float2 a, float2 b) { return __fadd2_rn(a, b); }
template <> __device__ __forceinline__ float2 csub<float2>(float2 a, float2 b) {
  return __fadd2_rn(a, make_float2(-b.x, -b.y));
}
template <> __device__ __forceinline__ float2 cmul<float2>(float2 a, float2 b) {
  const float2 t = __fmul2_rn(make_float2(a.y, a.y), make_float2(b.y, b.x));    // (ay by, ay bx)
  return __ffma2_rn(make_float2(a.x, a.x), b, make_float2(-t.x, t.y));         // (ax bx - ay by, ax by + ay bx)
}
// multiply by -i (forward) or +i (inverse)
template <typename C> __device__ __forceinline__ C cmul_mi(C a, bool inv) {
  C c; if (inv) { c.x = -a.y; c.y = a.x; } else { c.x = a.y; c.y = -a.x; } return c;
}
template <typename C, typename T> __device__ __forceinline__ C cscale(C a, T s) { a.x *= s; a.y *= s; return a; }

// --------------------------------------------------------------------------- batched copies
// for (i = tid; i < count; i += nthr) st(i, ld(i)), with UNR loads issued before their stores so a
// thread keeps UNR global reads in flight (a plain loop waits for each load before the next,
// because the stores in between may alias the next load's address).
template <int UNR, typename Ld, typename St>
__device__ __forceinline__ void batched_copy(int tid, int nthr, int count, Ld ld, St st) {
  using V = decltype(ld(0));
  for (int i0 = tid; i0 < count; i0 += UNR * nthr) {
    V v[UNR];
#pragma unroll
    for (int u = 0; u < UNR; ++u) {
      const int i = i0 + u * nthr;
      if (i < count) v[u] = ld(i);
    }
#pragma unroll
    for (int u = 0; u < UNR; ++u) {
      const int i = i0 + u * nthr;
      if (i < count) st(i, v[u]);
    }
  }
}

// --------------------------------------------------------------------------- per-load solver scalars
// One record per load, updated only by the last block of the kernel that owns the quantity.
struct LoadScalars {
  double rz;        // r . M^-1 r of the current recurrence
  double beta;      // CG direction update coefficient
  double alpha;     // CG step of the last apply
  double target2;   // squared absolute stopping threshold
  double norm;      // ||f||
  double absolute;  // certified ||f - K u||
  double res2;      // recurrence ||r||^2
  double mean_r[3]; // mean of r over nodes (projection P)
  double mean_z[3]; // mean of s.w over nodes (projection P of the preconditioned residual)
  double mean_u[3]; // mean of u over nodes (certification projection)
  int active;       // recurrence still iterating
  int bad;          // non-finite / non-positive curvature latch
  int failed;       // set by the apply finalizer when p.q or rz is invalid
  int iterations;   // PCG iterations taken
  int touched;      // mixed refinement: this load ran an inner solve in the current sweep
  int reliable;     // mixed: replace the FP32 recurrence residual by the FP64 true residual now
  double anchor;    // mixed: recurrence ||r||^2 at the last true-residual replacement
  int total_iterations;  // mixed refinement: inner iterations summed over sweeps
  int frozen;       // batched contexts: this load's design took its last attempt (later attempts skip it)
  int restarts;     // restarts taken by this load's design
  double rz_cross;  // flexible beta: new residual . previous preconditioned residual
  int ticket[8];    // per-kernel block tickets for the last-block finalizers
};

enum Ticket { kTicketApply = 0, kTicketUpdate = 1, kTicketFZ = 2, kTicketIFX = 3, kTicketAux = 4, kTicketAux2 = 5 };

__device__ __forceinline__ int flat_tid() {
  return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
}
__device__ __forceinline__ int block_threads() { return blockDim.x * blockDim.y * blockDim.z; }

// Returns true in exactly one block per load: the last one to arrive. Every block that calls it
// must have written its partials first. Resets the ticket for the next launch.
__device__ __forceinline__ bool last_block(int* ticket, int nblocks) {
  __shared__ int amlast;
  __syncthreads();
  if (flat_tid() == 0) {
    __threadfence();
    int t = atomicAdd(ticket, 1);
    amlast = (t == nblocks - 1);
    if (amlast) *ticket = 0;
  }
  __syncthreads();
  if (amlast) __threadfence();
  return amlast;
}

// Sum over the lanes of a warp that may be partial (the last warp of a block whose size is not a
// multiple of 32): `active` lanes take part, lane 0 receives the sum.
__device__ __forceinline__ double warp_reduce(double v, int lane, int active) {
  if (active >= 32) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  } else {
    const unsigned mask = (1u << active) - 1u;
    for (int o = 16; o > 0; o >>= 1) {
      const double t = __shfl_down_sync(mask, v, o);
      if (lane + o < active) v += t;
    }
  }
  return v;
}

// Block-wide sum of NV doubles for any block size; result valid in thread 0. Uses `red`
// (>= NV * 32 doubles).
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* red) {
  const int tid = flat_tid();
  const int nthreads = block_threads();
  const int warp = tid >> 5, lane = tid & 31, nwarps = (nthreads + 31) >> 5;
  const int active = min(32, nthreads - (warp << 5));
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = warp_reduce(v[k], lane, active);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) red[k * 32 + warp] = v[k];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double s = lane < nwarps ? red[k * 32 + lane] : 0.0;
      v[k] = warp_reduce(s, lane, active);
    }
  }
}

// Fixed-order sum of `count` partials by the first warp of the block (which may be partial);
// call from every thread with tid < 32; result in thread 0.
__device__ __forceinline__ double warp_sum_partials(const double* p, int count) {
  const int tid = flat_tid();
  const int active = min(32, block_threads());
  double s = 0.0;
  for (int i = tid; i < count; i += active) s += __ldcg(p + i);
  return warp_reduce(s, tid, active);
}

// --------------------------------------------------------------------------- operator constants
// Per unit of a: cst = g^2 V = h/16 folded with the isotropic medium and the Gauss weights
// (1 for the constant strain modes, 1/3 for the linear ones, 1/9 for the bilinear ones).
struct OpConst {
  double l0, m0;      // cst * lambda, cst * mu
  double l1, m1, n1;  // cst * lambda/3, cst * mu/3, cst * (lambda + 3 mu)/3
  double k7;          // cst * (lambda + 4 mu)/9
};

inline OpConst make_opconst(int n, double lam, double mu) {
  const double h = 1.0 / n, cst = h / 16.0;
  OpConst c;
  c.l0 = cst * lam; c.m0 = cst * mu;
  c.l1 = cst * lam / 3.0; c.m1 = cst * mu / 3.0; c.n1 = cst * (lam + 3.0 * mu) / 3.0;
  c.k7 = cst * (lam + 4.0 * mu) / 9.0;
  return c;
}

// Element action in modal form. Q[m][c] is the Hadamard (sum/difference) transform of the 8
// nodal displacements along x (bit 0 of m), y (bit 1), z (bit 2); P[m][c] is the transform of
// the nodal forces, f = sum_m s(m,b) P[m]. The constant mode carries no strain: P[0] = 0.
// This is the exact 2x2x2-Gauss HEX8 product for C = A * C0(lambda, mu), with the strain /
// stress / B^T steps of the element collapsed algebraically for an isotropic medium.
template <typename T>
__host__ __device__ __forceinline__ void element_modal(const T (&Q)[8][3], T A, const OpConst& k, T (&P)[8][3]) {
  // constant strain modes (weight 1)
  const T l0 = A * T(k.l0), m0 = A * T(k.m0);
  const T m20 = m0 + m0;
  const T tr = Q[1][0] + Q[2][1] + Q[4][2];
  const T lt = l0 * tr;
  const T gyz = m0 * (Q[4][1] + Q[2][2]);
  const T gxz = m0 * (Q[4][0] + Q[1][2]);
  const T gxy = m0 * (Q[2][0] + Q[1][1]);
  P[1][0] = fma(m20, Q[1][0], lt); P[1][1] = gxy; P[1][2] = gxz;
  P[2][0] = gxy; P[2][1] = fma(m20, Q[2][1], lt); P[2][2] = gyz;
  P[4][0] = gxz; P[4][1] = gyz; P[4][2] = fma(m20, Q[4][2], lt);
  // linear strain modes (weight 1/3)
  const T l1 = A * T(k.l1), m1 = A * T(k.m1), n1 = A * T(k.n1);
  P[3][0] = fma(n1, Q[3][0], l1 * Q[6][2]);
  P[3][1] = fma(n1, Q[3][1], l1 * Q[5][2]);
  P[5][0] = fma(n1, Q[5][0], l1 * Q[6][1]);
  P[5][2] = fma(n1, Q[5][2], l1 * Q[3][1]);
  P[6][1] = fma(n1, Q[6][1], l1 * Q[5][0]);
  P[6][2] = fma(n1, Q[6][2], l1 * Q[3][0]);
  const T S = Q[3][2] + Q[5][1] + Q[6][0];
  P[3][2] = m1 * (S + Q[3][2]);
  P[5][1] = m1 * (S + Q[5][1]);
  P[6][0] = m1 * (S + Q[6][0]);
  // bilinear strain modes (weight 1/9)
  const T k7 = A * T(k.k7);
  P[7][0] = k7 * Q[7][0]; P[7][1] = k7 * Q[7][1]; P[7][2] = k7 * Q[7][2];
  P[0][0] = T(0); P[0][1] = T(0); P[0][2] = T(0);
}

// 8 nodal values (b = bx + 2by + 4bz) -> modal Q[m]; all 8 modes.
template <typename T>
__host__ __device__ __forceinline__ void hadamard8(const T (&v)[8][3], T (&Q)[8][3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    T s[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) s[i] = v[i][c];
    // x level (bit 0)
#pragma unroll
    for (int i = 0; i < 8; i += 2) { T a = s[i], b = s[i + 1]; s[i] = b + a; s[i + 1] = b - a; }
    // y level (bit 1)
#pragma unroll
    for (int i = 0; i < 8; ++i) if (!(i & 2)) { T a = s[i], b = s[i + 2]; s[i] = b + a; s[i + 2] = b - a; }
    // z level (bit 2)
#pragma unroll
    for (int i = 0; i < 4; ++i) { T a = s[i], b = s[i + 4]; s[i] = b + a; s[i + 4] = b - a; }
#pragma unroll
    for (int i = 0; i < 8; ++i) Q[i][c] = s[i];
  }
}

}  // namespace pgj
