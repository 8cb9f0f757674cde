// Slab-fused PCG iteration: the vector updates of the recurrence fused with the x/y transforms of
// the Green apply, so that one iteration is four kernels over the DOF vectors and the spectrum:
//
//   operator : q = K p, alpha = rz / p.q                         (pgj_operator.cu)
//   fxy      : u += alpha p, r -= alpha q, ||r||^2, sum r  -> last block: masks, mean r;
//              2D real DFT over (x, y) of s.r for one (load, component, z) slab    (this file)
//   fz       : DFT along z, - mean r . DFT(s), symbol, <v, G v> and mean(s.w) by Parseval,
//              inverse along z -> last block: rz, beta, mean(s.w)                   (pgj_fft.cu)
//   ifxy     : inverse y and C2R x of the slab, p = (s.w - mean(s.w)) + beta p      (this file)
//
// Same recurrence as resident.py:119-131 of exp/asg_gpu_resident_20261103 (the unfused kernels in
// pgj_pcg.cu and the five-pass Green apply in pgj_fft.cu do it step by step); the two means of the
// projection P are exact linear identities moved into the spectral pass:
//   DFT(s.(r - m)) = DFT(s.r) - m DFT(s),   sum_x s.w = sum_k W(k) conj(DFT(s)(k)).
// A block owns one component of one z-plane: an n x n real slab, two rows packed per complex
// line for the real transform (lines at an odd pitch of n + 1 complex values, so that a warp
// working on 32 lines at the same index touches distinct banks), the half spectrum as n rows of
// nsp (even) complex values.
#include "pgj_fft_engine.cuh"
#include <cstdlib>
#include <cstring>
#include <type_traits>

namespace pgj {

enum SlabMode { kSlabUpdate = 0, kSlabInit = 1, kSlabSync = 2 };

struct SlabArgs {
  int n, ns, nsp;
  FFTPlan plan;
  FastDiv div_n, div_ns, div_nh;  // n, ns, n / 2
  void* p;                // (L,3N) T search directions
  const void* q;          // (L,3N) T K p
  void* r;                // (L,3N) T recurrence residual
  void* u;                // (L,3N) U iterate (FP64 x, or the FP32 correction d)
  const double* r64;      // sync mode: FP64 true residual
  const double* scale;    // (designs, 3N) FP64 scale field s
  const float* scale32;   // FP32 contexts: (designs, 3, N) component-planar FP32 copy of s
  void* spec;             // (L,3,n,n,nsp) complex T
  void* zprev;            // flexible beta: (L,3N) T preconditioned residual of the previous direction
  int flex;               // flexible beta: fxy sums r_new . z_prev, ifxy stores z
  const void* tw;         // n complex T twiddles
  LoadScalars* scal;      // recurrence records
  const LoadScalars* out; // sync mode: certificate records (res2, mean r of the true residual)
  double* partials;
  int cap;
  double rel_delta2;
  int loads;
  int lpd;                // loads per design: load l uses the scale field of design l / lpd
  int init;               // ifxy: p = P(s.w) (first direction)
  int set_cond;           // ifxy: set the WHILE condition (any load active, bounded body count)
  cudaGraphConditionalHandle h;
  int* counters;
  // The halo-free operator's boundary rows reach the update (k_fxy, update mode) through fields the
  // update does not use otherwise: r64 (the sync mode's FP64 residual) carries qb, (L, n, ntiles, 3, n),
  // init the tile height and set_cond the tile count. Four more fields in this parameter block (which
  // the kernels copy to local memory) had made the generic FP32 update twice as slow at n = 48.
};

// the loop body runs at most cap + 100 times per attempt (the same bound as the unfused loop body)

template <typename T>
__device__ __forceinline__ T* real_view(cplx<T>* b) { return reinterpret_cast<T*>(b); }

// n = 64: a 64-point line as an 8 x 8 four-step transform held by 8 lanes (lane t holds points
// t + 8b), with the transpose through the line's own shared-memory region L (rows of 9, 72 slots).
// Forward from registers v[b] = x[t + 8b]: on return v[k1] = X[t + 8 k1]. Inverse from
// v[k1] = X[t + 8 k1]: on return v[b] = x[t + 8 b] (unnormalised). The caller's eight lanes of the
// line must be converged; L must not be read by other lanes meanwhile.
// 72 slots: two lines that share a half-warp (FP32 complex values are 8 bytes, 16 lanes per
// shared-memory pass) then sit 16 banks apart, so both the row and the column accesses of the
// transpose are free of bank conflicts.
constexpr int kLine64 = 72;
template <typename T>
__device__ __forceinline__ void line64(cplx<T> (&v)[8], cplx<T>* L, int t, const cplx<T>* __restrict__ tw, bool inv) {
  using C = cplx<T>;
  Radix<T, 8>::run(v, inv);
#pragma unroll
  for (int k = 1; k < 8; ++k) {
    C w = __ldg(&tw[t * k]);
    if (inv) w.y = -w.y;
    v[k] = cmul(v[k], w);
  }
  __syncwarp();
#pragma unroll
  for (int k = 0; k < 8; ++k) L[k * 9 + t] = v[k];
  __syncwarp();
#pragma unroll
  for (int j = 0; j < 8; ++j) v[j] = L[t * 9 + j];
  Radix<T, 8>::run(v, inv);
  __syncwarp();
}

// ------------------------------------------------------------------------------------------ fxy
// W4: blocks of at most 288 threads, four resident per SM (56 registers); otherwise up to 512
// threads, two per SM.
// R64 (n = 64, 288 threads): x and y lines as register four-step transforms (line64); shared
// memory holds 36 lines of 72 complex values (packed x lines, then per-warp transpose space) and
// the n x nsp half-spectrum rows.
// FLEX: the flexible direction update (FP32 only) adds r_new . z_prev to the block sums; a separate
// instantiation, so the plain forms keep their register budget (the runtime branch cost 3-6 us).
// HFQ (FP32 update mode): q comes from the halo-free operator, whose first rows of every tile
// (y % hf_ty == 0) lack the contributions of the element row below; those are in qb and added here.
template <typename T, typename U, int MODE, bool W4, bool R64, bool FLEX = false, bool HFQ = false>
__global__ void __launch_bounds__(W4 ? 288 : 512, W4 ? 4 : 2) k_fxy(const SlabArgs A) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int c = blockIdx.x, z = blockIdx.y, load = blockIdx.z;
  LoadScalars& S = A.scal[load];
  if (MODE == kSlabSync ? (S.reliable == 0) : (S.active == 0)) return;
  const int n = A.n, ns = A.ns, nsp = A.nsp;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int nn = n * n;
  C* b0 = reinterpret_cast<C*>(smem_raw);
  C* b1 = b0 + (R64 ? 36 * kLine64 : size_t(n) * nsp);
  double* red = reinterpret_cast<double*>(b1 + size_t(n) * nsp);
  const size_t N = size_t(nn) * n, N3 = 3 * N;
  const size_t node0 = size_t(z) * nn;
  // FP32 recurrence vectors r, d and q are component-planar, (3, N) per load: the slab's values are
  // contiguous; the direction p (the operator's input, staged by rows) and the FP64 vectors (the FP64
  // true residual included) keep the node-major interleaved layout
  constexpr bool PL = sizeof(T) == 4;
  constexpr int KS = PL ? 1 : 3;                           // element stride of consecutive nodes
  const size_t off = PL ? size_t(load) * N3 + size_t(c) * N + node0
                        : size_t(load) * N3 + 3 * node0 + c;  // dof of node (0,0,z), component c
  const size_t off64 = size_t(load) * N3 + 3 * node0 + c;
  T* r = reinterpret_cast<T*>(A.r) + off;
  const size_t dsg = size_t(load / A.lpd);
  const double* sc = A.scale + dsg * N3 + 3 * node0 + c;
  const float* s32 = sizeof(T) == 4 ? A.scale32 + dsg * N3 + size_t(c) * nn * n + node0 : nullptr;  // coalesced
  T* packed = real_view<T>(b0);
  const int lpx = R64 ? kLine64 : n + 1;  // pitch of the packed x lines
  double acc[FLEX ? 3 : 2] = {};
  const double alpha = MODE == kSlabUpdate ? S.alpha : 0.0;
  const T a = T(alpha);
  // nodes whose loads are in flight together (the FP64 update keeps five doubles per node)
  constexpr int UNR = (MODE == kSlabUpdate && sizeof(T) == 8) ? 2 : 4;
  const T* pg = reinterpret_cast<const T*>(A.p) + off64;  // interleaved: stride 3
  const T* qg = reinterpret_cast<const T*>(A.q) + off;
  const T* zg = FLEX ? reinterpret_cast<const T*>(A.zprev) + off : nullptr;
  U* ug = reinterpret_cast<U*>(A.u) + off;
  const double* r64 = A.r64 + off64;
  // The halo-free operator leaves the first row of every tile (y % hf_ty == 0) without the
  // contributions of the element row below; those are in qb. With HFQ the update runs in two passes:
  // the other rows first (a cheap row test per node), then the first rows with q + qb (reading qb
  // per node in one pass measured 7 us slower, staging it in shared memory behind a barrier 9 us).
  if constexpr (HFQ) {
    // the lambdas live only in this branch: capturing the update's locals by reference elsewhere put
    // them in local memory and doubled the generic slab update (n = 48: 78.8 vs 40.0 us)
    const int hf_ty = A.init, hf_ntiles = A.set_cond;
    const T* qbb = reinterpret_cast<const T*>(A.r64) + ((size_t(load) * n + z) * hf_ntiles * 3 + c) * size_t(n);
    const int hshift = (hf_ty & (hf_ty - 1)) == 0 ? __ffs(hf_ty) - 1 : -1;
    auto first_row = [&](int i) -> bool {
      if constexpr (!HFQ) return false;
      const int yy = R64 ? (i >> 6) : fdiv(i, A.div_n);
      if (hshift >= 0) return (yy & ((1 << hshift) - 1)) == 0;
      return (yy / hf_ty) * hf_ty == yy;
    };
    // count nodes, node index i = idx(e), BND: the first rows (q + qb)
    auto pass = [&](int count, auto idx, auto bnd_tag) {
      constexpr bool BND = decltype(bnd_tag)::value;
      for (int e0 = tid; e0 < count; e0 += UNR * nthr) {
        // all loads of UNR nodes first, then the updates and stores
        T pv[UNR], qv[UNR], rv[UNR];
        U uv[UNR];
        double sv[UNR];
        bool on[UNR];
  #pragma unroll
        for (int j = 0; j < UNR; ++j) {
          const int e = e0 + j * nthr;
          on[j] = e < count;
          if (!on[j]) continue;
          const int i = idx(e);
          if (!BND && first_row(i)) { on[j] = false; continue; }
          const size_t k = size_t(KS) * i;
          sv[j] = sizeof(T) == 4 ? double(s32[i]) : sc[3 * size_t(i)];
          if (MODE == kSlabUpdate) {
            pv[j] = pg[3 * size_t(i)]; qv[j] = qg[k]; rv[j] = r[k]; uv[j] = ug[k];
            if constexpr (BND) {
              const int t = R64 ? (i >> (6 + hshift)) : fdiv(i, A.div_n) / hf_ty;
              qv[j] += qbb[t * 3 * n + (i - t * hf_ty * n)];
            }
          } else if (MODE == kSlabSync) {
            rv[j] = T(r64[3 * size_t(i)]);
          } else {
            rv[j] = r[k];
          }
        }
  #pragma unroll
        for (int j = 0; j < UNR; ++j) {
          if (!on[j]) continue;
          const int i = idx(e0 + j * nthr);
          const size_t k = size_t(KS) * i;
          const int y = fdiv(i, A.div_n), x = i - y * n;
          T rj = rv[j];
          if (MODE == kSlabUpdate) {
            ug[k] = uv[j] + U(alpha) * U(pv[j]);
            rj = rj - a * qv[j];
            r[k] = rj;
            const double rd = double(rj);
            acc[0] += rd * rd;
            acc[1] += rd;
            if constexpr (FLEX) acc[FLEX ? 2 : 0] += rd * double(zg[k]);
          } else if (MODE == kSlabSync) {
            r[k] = rj;
          }
          // rows 2l and 2l+1 packed as the real and imaginary parts of complex line l
          packed[2 * ((y >> 1) * lpx + x) + (y & 1)] = T(sv[j]) * rj;
        }
      }
    };
    pass(nn, [](int e) { return e; }, std::false_type{});
    // the first rows: e = (tile, x) -> node (tile * hf_ty, x)
    pass(hf_ntiles * n, [&](int e) {
      const int t = R64 ? (e >> 6) : fdiv(e, A.div_n);
      return t * hf_ty * n + (e - t * n);
    }, std::true_type{});
  } else {
    for (int i0 = tid; i0 < nn; i0 += UNR * nthr) {
      // all loads of UNR nodes first, then the updates and stores
      T pv[UNR], qv[UNR], rv[UNR];
      U uv[UNR];
      double sv[UNR];
#pragma unroll
      for (int j = 0; j < UNR; ++j) {
        const int i = i0 + j * nthr;
        if (i < nn) {
          const size_t k = size_t(KS) * i;
          sv[j] = sizeof(T) == 4 ? double(s32[i]) : sc[3 * size_t(i)];
          if (MODE == kSlabUpdate) { pv[j] = pg[3 * size_t(i)]; qv[j] = qg[k]; rv[j] = r[k]; uv[j] = ug[k]; }
          else if (MODE == kSlabSync) rv[j] = T(r64[3 * size_t(i)]);
          else rv[j] = r[k];
        }
      }
#pragma unroll
      for (int j = 0; j < UNR; ++j) {
        const int i = i0 + j * nthr;
        if (i < nn) {
          const size_t k = size_t(KS) * i;
          const int y = fdiv(i, A.div_n), x = i - y * n;
          T rj = rv[j];
          if (MODE == kSlabUpdate) {
            ug[k] = uv[j] + U(alpha) * U(pv[j]);
            rj = rj - a * qv[j];
            r[k] = rj;
            const double rd = double(rj);
            acc[0] += rd * rd;
            acc[1] += rd;
            if constexpr (FLEX) acc[FLEX ? 2 : 0] += rd * double(zg[k]);
          } else if (MODE == kSlabSync) {
            r[k] = rj;
          }
          // rows 2l and 2l+1 packed as the real and imaginary parts of complex line l
          packed[2 * ((y >> 1) * lpx + x) + (y & 1)] = T(sv[j]) * rj;
        }
      }
    }
  }
  __syncthreads();
  const C* tw = reinterpret_cast<const C*>(A.tw);
  C* res;
  C* oth;
  const int warp = tid >> 5, li = (tid & 31) >> 3, t8 = tid & 7;
  if constexpr (R64) {
    if (warp < 8) {  // 32 packed x lines, four per warp, eight lanes per line
      C* L = b0 + (4 * warp + li) * kLine64;
      C v[8];
#pragma unroll
      for (int b = 0; b < 8; ++b) v[b] = L[t8 + 8 * b];
      line64<T>(v, L, t8, tw, false);
#pragma unroll
      for (int k1 = 0; k1 < 8; ++k1) L[t8 + 8 * k1] = v[k1];
    }
    __syncthreads();
    res = b0;
    oth = b1;
  } else {
    res = fft_lines<T, true>(b0, b1, n / 2, lpx, 1, A.plan, A.div_nh, tw, false, tid, nthr);
    oth = res == b0 ? b1 : b0;
  }
  // split the packed transforms: row rho = 2l (real part) and 2l+1 (imaginary part)
  for (int i = tid; i < n * ns; i += nthr) {
    const int rho = fdiv(i, A.div_ns), k = i - rho * ns;
    const C* line = res + (rho >> 1) * lpx;
    const C zk = line[k];
    const C zn = line[k == 0 ? 0 : n - k];
    C o;
    if ((rho & 1) == 0) { o.x = T(0.5) * (zk.x + zn.x); o.y = T(0.5) * (zk.y - zn.y); }
    else { o.x = T(0.5) * (zk.y + zn.y); o.y = T(0.5) * (zn.x - zk.x); }
    oth[rho * nsp + k] = o;
  }
  __syncthreads();
  // y transform of the ns columns
  C* sp = reinterpret_cast<C*>(A.spec) + ((size_t(load) * 3 + c) * n + z) * size_t(n) * nsp;
  if constexpr (R64) {
    // columns four per warp (nine warps), straight from the rows to the spectrum in global memory
    // (staging the plane for one bulk store measured slower: 99 vs 93 us FP64, 51 vs 47 us FP32)
    const int col = 4 * warp + li;
    const bool valid = col < ns;
    C* L = b0 + (4 * warp + li) * kLine64;  // free once the split has read the packed lines
    C v[8];
    const C zero = cmk<C>(0.0, 0.0);
#pragma unroll
    for (int b = 0; b < 8; ++b) v[b] = valid ? oth[(t8 + 8 * b) * nsp + col] : zero;
    line64<T>(v, L, t8, tw, false);
    if (valid) {
#pragma unroll
      for (int k1 = 0; k1 < 8; ++k1) sp[size_t(t8 + 8 * k1) * nsp + col] = v[k1];
    }
  } else {
    C* res2 = fft_lines<T, true>(oth, res, ns, 1, nsp, A.plan, A.div_ns, tw, false, tid, nthr);
    for (int i = tid; i < n * ns; i += nthr) {
      const int ky = fdiv(i, A.div_ns), kx = i - ky * ns;
      sp[size_t(ky) * nsp + kx] = res2[ky * nsp + kx];
    }
  }
  if (MODE == kSlabInit) return;

  const int nblk = 3 * n, blk = c + 3 * z;
  double* part = A.partials + size_t(load) * kPartialQ * kMaxPartials;
  if (MODE == kSlabUpdate) {
    block_sum<FLEX ? 3 : 2>(acc, red);
    if (tid == 0) {
      part[blk] = acc[0];
      for (int cc = 0; cc < 3; ++cc) part[(1 + cc) * kMaxPartials + blk] = cc == c ? acc[1] : 0.0;
      if constexpr (FLEX) part[4 * kMaxPartials + blk] = acc[FLEX ? 2 : 0];
    }
    if (!last_block(&S.ticket[kTicketUpdate], nblk)) return;
    if (tid < 32) {
      constexpr int NV = FLEX ? 5 : 4;
      double v[5] = {};
      for (int k = 0; k < NV; ++k) v[k] = warp_sum_partials(part + k * kMaxPartials, nblk);
      if (tid == 0) {
        if constexpr (FLEX) S.rz_cross = v[4];
        // same bookkeeping as the unfused update (k_update_ur)
        const double res2 = v[0];
        const bool finite = isfinite(res2);
        const int it = S.iterations + 1;
        const bool valid = S.failed == 0;
        const bool keep = valid && finite && (res2 > S.target2) && (it < A.cap);
        S.iterations = it;
        S.bad = S.bad | (valid ? 0 : 1) | (finite ? 0 : 1);
        S.active = keep ? 1 : 0;
        S.res2 = res2;
        for (int cc = 0; cc < 3; ++cc) S.mean_r[cc] = v[1 + cc] / double(N);
        if (A.rel_delta2 > 0.0) {
          const bool ok = valid && finite && it < A.cap;
          S.reliable = ok && ((keep && res2 < A.rel_delta2 * S.anchor) || (!keep && res2 <= S.target2)) ? 1 : 0;
        }
      }
    }
  } else {  // kSlabSync: the recurrence restarts from the FP64 true residual (k_rel_sync)
    if (!last_block(&S.ticket[kTicketAux2], nblk)) return;
    if (tid == 0) {
      const LoadScalars& O = A.out[load];
      S.res2 = O.res2;
      S.anchor = O.res2;
      for (int cc = 0; cc < 3; ++cc) S.mean_r[cc] = O.mean_r[cc];
      S.active = isfinite(O.res2) && O.res2 > S.target2 && S.iterations < A.cap && !S.bad ? 1 : 0;
      S.reliable = 0;
    }
  }
}

// ----------------------------------------------------------------------------------------- ifxy
template <typename T, bool W4, bool R64, bool FLEX = false>
__global__ void __launch_bounds__(W4 ? 288 : 512, W4 ? 4 : 2) k_ifxy(const SlabArgs A) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int c = blockIdx.x, z = blockIdx.y, load = blockIdx.z;
  const int tid = threadIdx.x, nthr = blockDim.x;
  if (A.set_cond && c == 0 && z == 0 && load == 0 && tid == 0) {
    int any = 0;
    for (int l = 0; l < A.loads; ++l) any |= A.scal[l].active;
    const int runs = ++A.counters[0];
    A.counters[5] += 1;                                 // loop bodies over the whole solve
    if (runs >= A.cap + 100) A.counters[1] = 1;  // recorded: loop stopped by the bound
    cudaGraphSetConditional(A.h, (any && runs < A.cap + 100) ? 1u : 0u);
  }
  const LoadScalars& S = A.scal[load];
  if (!S.active) return;
  const int n = A.n, ns = A.ns, nsp = A.nsp;
  const int nn = n * n;
  const int lpx = R64 ? kLine64 : n + 1;  // pitch of the packed x lines
  C* b0 = reinterpret_cast<C*>(smem_raw);
  C* b1 = b0 + (R64 ? 36 * kLine64 : size_t(n) * nsp);
  const C* sp = reinterpret_cast<const C*>(A.spec) + ((size_t(load) * 3 + c) * n + z) * size_t(n) * nsp;
  const C* tw = reinterpret_cast<const C*>(A.tw);
  const int warp = tid >> 5, li = (tid & 31) >> 3, t8 = tid & 7;
  C* res;
  C* oth;
  if constexpr (R64) {
    // inverse y of four columns per warp into the rows (b1). FP64: the slab's half spectrum (n rows
    // of nsp, contiguous in global memory) first arrives in b1 as one bulk copy (56 vs 58 us); FP32
    // reads the columns straight from global memory (31 vs 33 us)
    constexpr bool kBulk = sizeof(T) == 8;
    __shared__ alignas(8) uint64_t sbar;
    if (kBulk) {
      if (tid == 0) {
        mbar_init(&sbar, 1);
        fence_mbar_init();
      }
      __syncthreads();
      if (tid == 0) {
        const unsigned pbytes = unsigned(size_t(n) * nsp * sizeof(C));
        mbar_expect_tx(&sbar, pbytes);
        tma_row(b1, sp, pbytes, &sbar);
      }
      const bool arrived = mbar_wait(&sbar, 0);  // bounded; every thread observes the arrival
      if (__syncthreads_or(!arrived)) {
        if (tid == 0) atomicExch(&A.counters[2], 1);  // reported as PGJ_ERR_TIMEOUT
        return;
      }
    }
    const C* src = kBulk ? b1 : sp;
    const int col = 4 * warp + li;
    const bool valid = col < ns;
    C* L = b0 + (4 * warp + li) * kLine64;
    C v[8];
    const C zero = cmk<C>(0.0, 0.0);
#pragma unroll
    for (int k1 = 0; k1 < 8; ++k1) v[k1] = valid ? src[(t8 + 8 * k1) * nsp + col] : zero;
    line64<T>(v, L, t8, tw, true);  // its warp barriers order the column reads before the writes
    if (valid) {
#pragma unroll
      for (int b = 0; b < 8; ++b) b1[(t8 + 8 * b) * nsp + col] = v[b];
    }
    __syncthreads();
    res = b1;
    oth = b0;
  } else {
    batched_copy<8>(tid, nthr, n * ns, [&](int i) {
      const int ky = fdiv(i, A.div_ns), kx = i - ky * ns;
      return sp[size_t(ky) * nsp + kx];
    }, [&](int i, C v) {
      const int ky = fdiv(i, A.div_ns), kx = i - ky * ns;
      b0[ky * nsp + kx] = v;
    });
    __syncthreads();
    res = fft_lines<T, true>(b0, b1, ns, 1, nsp, A.plan, A.div_ns, tw, true, tid, nthr);
    oth = res == b0 ? b1 : b0;
  }
  // C2R packing: line l = A + i B over the full x range (rows 2l, 2l+1 Hermitian-extended,
  // imaginary parts of the DC and Nyquist bins dropped)
  for (int i = tid; i < (n / 2) * n; i += nthr) {
    const int l = fdiv(i, A.div_n), k = i - l * n;
    C v[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const C* row = res + (2 * l + h) * nsp;
      C val;
      if (k < ns) {
        val = row[k];
        if (k == 0 || k == n / 2) val.y = T(0);
      } else {
        val = cconj(row[n - k]);
      }
      v[h] = val;
    }
    C zz;
    zz.x = v[0].x - v[1].y;
    zz.y = v[0].y + v[1].x;
    oth[l * lpx + k] = zz;
  }
  __syncthreads();
  C* res2;
  if constexpr (R64) {
    if (warp < 8) {
      C* L = oth + (4 * warp + li) * kLine64;
      C v[8];
#pragma unroll
      for (int k1 = 0; k1 < 8; ++k1) v[k1] = L[t8 + 8 * k1];
      line64<T>(v, L, t8, tw, true);
#pragma unroll
      for (int b = 0; b < 8; ++b) L[t8 + 8 * b] = v[b];
    }
    __syncthreads();
    res2 = oth;
  } else {
    res2 = fft_lines<T, true>(oth, res, n / 2, lpx, 1, A.plan, A.div_nh, tw, true, tid, nthr);
  }
  const T* wv = real_view<T>(res2);
  const size_t node0 = size_t(z) * nn;
  constexpr bool PL = sizeof(T) == 4;  // FP32 recurrence vectors other than p are component-planar
  constexpr int KS = PL ? 1 : 3;
  const size_t N = size_t(nn) * n;
  const size_t off = PL ? size_t(load) * 3 * N + size_t(c) * N + node0 : size_t(load) * 3 * N + 3 * node0 + c;
  T* p = reinterpret_cast<T*>(A.p) + (size_t(load) * 3 * N + 3 * node0 + c);  // interleaved: stride 3
  const size_t dsg = size_t(load / A.lpd) * 3 * size_t(nn) * n;  // this load's design
  const double* sc = A.scale + dsg + 3 * node0 + c;
  const float* s32 = sizeof(T) == 4 ? A.scale32 + dsg + size_t(c) * nn * n + node0 : nullptr;  // coalesced
  const T m = T(S.mean_z[c]);
  const T beta = T(S.beta);
  constexpr int UNR = 4;
  for (int i0 = tid; i0 < nn; i0 += UNR * nthr) {
    T pv[UNR];
    double sv[UNR];
#pragma unroll
    for (int j = 0; j < UNR; ++j) {
      const int i = i0 + j * nthr;
      if (i < nn) {
        sv[j] = sizeof(T) == 4 ? double(s32[i]) : sc[3 * size_t(i)];
        pv[j] = A.init ? T(0) : p[3 * size_t(i)];
      }
    }
#pragma unroll
    for (int j = 0; j < UNR; ++j) {
      const int i = i0 + j * nthr;
      if (i < nn) {
        const int y = fdiv(i, A.div_n), x = i - y * n;
        const T w = wv[2 * ((y >> 1) * lpx + x) + (y & 1)];
        const T zv = T(sv[j]) * w - m;
        p[3 * size_t(i)] = A.init ? zv : zv + beta * pv[j];
        if constexpr (FLEX) reinterpret_cast<T*>(A.zprev)[off + size_t(KS) * i] = zv;
      }
    }
  }
}

// ------------------------------------------------------------------------------------ host side
static size_t slab_smem(int n, int nsp, size_t tsz) { return 2 * size_t(n) * nsp * 2 * tsz + 32 * 3 * 8 + 64; }
// R64: 36 lines of kLine64 complex values, then the n x nsp rows, then the reduction
static size_t slab_smem64(int nsp, size_t tsz) { return (36 * size_t(kLine64) + 64 * size_t(nsp)) * 2 * tsz + 32 * 3 * 8 + 64; }

static int slab_threads(const pgj_ctx* c) {
  int minr = 8;
  for (int i = 0; i < c->plan.nst; ++i) minr = c->plan.radix[i] < minr ? c->plan.radix[i] : minr;
  const int ns = c->ns;
  int w = (ns * c->n) / minr;  // butterflies of the widest stage over the y columns
  int t = ((w + 31) / 32) * 32;
  if (t > 512) t = 512;
  if (t < 64) t = 64;
  return t;
}

bool slab_fits_shape(int n, int prec) {
  const size_t tsz = prec == PGJ_FP32 ? 4 : 8;
  const int ns = n / 2 + 1, nsp = ns + (ns & 1);
  return slab_smem(n, nsp, tsz) <= 110 * 1024;  // two blocks per SM
}

bool slab_fits(const pgj_ctx* c) { return slab_fits_shape(c->n, c->prec); }

template <typename T, typename U, bool W4, bool R64, bool FLEX = false>
static void set_fxy_smem(int lim) {
  cudaFuncSetAttribute(k_fxy<T, U, kSlabUpdate, W4, R64, FLEX>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  if constexpr (sizeof(T) == 4 && R64)
    cudaFuncSetAttribute(k_fxy<T, U, kSlabUpdate, W4, R64, FLEX, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         lim);
  cudaFuncSetAttribute(k_fxy<T, U, kSlabInit, W4, R64, FLEX>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fxy<T, U, kSlabSync, W4, R64, FLEX>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_ifxy<T, W4, R64, FLEX>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
}

int prepare_slab_kernels() {
  const int lim = 112 * 1024;
  set_fxy_smem<double, double, false, false>(lim);
  set_fxy_smem<double, double, false, true>(lim);
  set_fxy_smem<float, float, false, false>(lim);
  set_fxy_smem<float, float, true, false>(lim);
  set_fxy_smem<float, float, true, true>(lim);
  set_fxy_smem<float, float, false, false, true>(lim);
  set_fxy_smem<float, float, true, false, true>(lim);
  set_fxy_smem<float, float, true, true, true>(lim);
  return check_launch();
}

// FP32 slabs of at most 288 threads take the four-per-SM register budget (PGJ_SLAB_W4=0: off)
static bool slab_w4(int prec, int thr) {
  const char* e = std::getenv("PGJ_SLAB_W4");
  return prec == PGJ_FP32 && thr <= 288 && !(e && e[0] == '0');
}

// n = 64 with 288 threads: register line transforms (PGJ_SLAB64=0: the generic passes)
static bool slab_r64(const pgj_ctx* c, int prec, int thr) {
  const char* e = std::getenv("PGJ_SLAB64");
  (void)prec;
  return c->n == 64 && thr == 288 && !(e && e[0] == '0');
}

bool slab_register_path(const pgj_ctx* c, int prec) { return slab_r64(c, prec, slab_threads(c)); }

static SlabArgs slab_args(pgj_ctx* c, int loads, int prec) {
  SlabArgs A;
  std::memset(&A, 0, sizeof(A));
  A.n = c->n; A.ns = c->ns; A.nsp = c->ns + (c->ns & 1);
  A.plan = c->plan;
  A.div_n = make_fastdiv(unsigned(c->n));
  A.div_ns = make_fastdiv(unsigned(c->ns));
  A.div_nh = make_fastdiv(unsigned(c->n / 2));
  A.p = c->p; A.q = c->q; A.r = c->r;
  A.r64 = c->r64; A.scale = c->scale; A.scale32 = c->scale32; A.spec = c->spec;
  A.flex = prec == PGJ_FP32 ? c->flex : 0;
  A.zprev = c->sw;  // unused by the fused form otherwise
  A.tw = prec == PGJ_FP32 ? static_cast<const void*>(static_cast<double2*>(c->tw) + c->n) : c->tw;
  A.scal = c->scal; A.out = c->scal_out; A.partials = c->partials;
  A.cap = c->cap; A.rel_delta2 = c->rel_delta2; A.loads = loads; A.lpd = c->lpd;
  A.counters = c->cond;
  return A;
}

// mode: kSlabUpdate (u in `u`: FP64 x, or the FP32 correction d), kSlabInit, kSlabSync
template <typename T, typename U, bool W4, bool R64, bool FLEX = false>
static void fxy_kernel(int mode, dim3 grid, int thr, size_t smem, cudaStream_t s, const SlabArgs& A) {
  switch (mode) {
    case kSlabUpdate:
      // the halo-free operator's consumer exists for the n = 64 register path only: compiled for the
      // generic paths as well, its instantiations made their plain update twice as slow (n = 48: 75.8
      // vs 39.9 us), though that code is not run there
      if constexpr (sizeof(T) == 4 && R64) {
        if (A.init) {
          k_fxy<T, U, kSlabUpdate, W4, R64, FLEX, true><<<grid, thr, smem, s>>>(A);
          break;
        }
      }
      k_fxy<T, U, kSlabUpdate, W4, R64, FLEX><<<grid, thr, smem, s>>>(A);
      break;
    case kSlabInit: k_fxy<T, U, kSlabInit, W4, R64, FLEX><<<grid, thr, smem, s>>>(A); break;
    default: k_fxy<T, U, kSlabSync, W4, R64, FLEX><<<grid, thr, smem, s>>>(A); break;
  }
}

int launch_fxy(pgj_ctx* c, int loads, int prec, int mode, void* u, cudaStream_t s) {
  SlabArgs A = slab_args(c, loads, prec);
  A.u = u;
  if (mode == kSlabUpdate && uses_hf(c, prec)) {  // q from the halo-free operator: add its boundary rows
    A.r64 = static_cast<const double*>(c->qb);  // the update mode's unused fields (see SlabArgs)
    A.init = c->hg.ty;
    A.set_cond = c->hg.ntiles;
  }
  const size_t tsz = prec == PGJ_FP32 ? 4 : 8;
  const dim3 grid(3, c->n, loads);
  const int thr = slab_threads(c);
  const bool r64 = slab_r64(c, prec, thr);
  const size_t smem = r64 ? slab_smem64(A.nsp, tsz) : slab_smem(A.n, A.nsp, tsz);
  if (prec == PGJ_FP32 && A.flex) {
    if (r64) fxy_kernel<float, float, true, true, true>(mode, grid, thr, smem, s, A);
    else if (slab_w4(prec, thr)) fxy_kernel<float, float, true, false, true>(mode, grid, thr, smem, s, A);
    else fxy_kernel<float, float, false, false, true>(mode, grid, thr, smem, s, A);
  } else if (prec == PGJ_FP32) {
    if (r64) fxy_kernel<float, float, true, true>(mode, grid, thr, smem, s, A);
    else if (slab_w4(prec, thr)) fxy_kernel<float, float, true, false>(mode, grid, thr, smem, s, A);
    else fxy_kernel<float, float, false, false>(mode, grid, thr, smem, s, A);
  } else {
    if (r64) fxy_kernel<double, double, false, true>(mode, grid, thr, smem, s, A);
    else fxy_kernel<double, double, false, false>(mode, grid, thr, smem, s, A);
  }
  return check_launch();
}

int launch_ifxy(pgj_ctx* c, int loads, int prec, bool init, cudaStream_t s, cudaGraphConditionalHandle h,
                bool set_cond) {
  SlabArgs A = slab_args(c, loads, prec);
  A.init = init ? 1 : 0;
  A.set_cond = set_cond ? 1 : 0;
  A.h = h;
  const size_t tsz = prec == PGJ_FP32 ? 4 : 8;
  const dim3 grid(3, c->n, loads);
  const int thr = slab_threads(c);
  const bool r64 = slab_r64(c, prec, thr);
  const size_t smem = r64 ? slab_smem64(A.nsp, tsz) : slab_smem(A.n, A.nsp, tsz);
  if (prec == PGJ_FP32 && A.flex) {
    if (r64) k_ifxy<float, true, true, true><<<grid, thr, smem, s>>>(A);
    else if (slab_w4(prec, thr)) k_ifxy<float, true, false, true><<<grid, thr, smem, s>>>(A);
    else k_ifxy<float, false, false, true><<<grid, thr, smem, s>>>(A);
  } else if (prec == PGJ_FP32) {
    if (r64) k_ifxy<float, true, true><<<grid, thr, smem, s>>>(A);
    else if (slab_w4(prec, thr)) k_ifxy<float, true, false><<<grid, thr, smem, s>>>(A);
    else k_ifxy<float, false, false><<<grid, thr, smem, s>>>(A);
  } else {
    if (r64) k_ifxy<double, false, true><<<grid, thr, smem, s>>>(A);
    else k_ifxy<double, false, false><<<grid, thr, smem, s>>>(A);
  }
  return check_launch();
}

}  // namespace pgj
