// Matrix-free periodic HEX8 operator, right-hand side, stiffness-diagonal scaling and projection.
//
// The operator q = K(a) p is a z-streaming stencil: a block owns full x-rows of n nodes and
// `ty` output node rows (plus one halo element row), and marches a chunk of z-planes. Node planes
// are staged in shared memory by bulk asynchronous copies (one row per copy, issued by the lanes
// of warp 0, 2-4 plane buffers, mbarrier completion; cp.async when rows are not 16-byte aligned).
// Each thread owns one element column. Per element plane it reads the four nodes of its upper face,
// forms the 2D Hadamard face modes, combines them with the lower face modes kept in registers
// (z-level), applies the modal element action, and splits the lower face into its four corner
// nodes: it keeps the (x, y) corner and hands the other three to their owners through a
// double-buffered exchange array, so one block barrier per plane publishes them. Fixed summation
// order: the result is deterministic (no atomics, unlike the reference's scatter in
// exp/asg_gpu_resident_20261103/scalar_fi.cu:14-36).
#include "pgj_internal.h"
#include <cmath>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

namespace pgj {

constexpr int kMaxPlaneStages = 4;  // node-plane buffers of the operator's staging pipeline (upper bound)

template <typename T> __device__ __forceinline__ void cp_async(T* dst, const T* src);
template <> __device__ __forceinline__ void cp_async<double>(double* dst, const double* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(dst)), "l"(src));
}
template <> __device__ __forceinline__ void cp_async<float>(float* dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(dst)), "l"(src));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }
__device__ __forceinline__ void cp_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::); }

// The rows of one plane issued by the lanes of one warp in parallel (lane r: rows r, r+32, ...):
// lane 0 arms the mbarrier for all rows first. Called by all 32 lanes of the warp. One copy per node
// row of 3n interleaved values, landing as [row][x][component]. (The component-planar FP32 vectors
// of slab-fused contexts are the recurrence's r, d and q; the operator's input p stays interleaved:
// staging a planar p as three component copies per plane measured 59.5 against 46.0 us.)
template <typename T>
__device__ __forceinline__ void tma_plane_warp(T* buf, const T* in, int pz, int y0, int rows, int n, uint64_t* bar,
                                               int lane) {
  const unsigned rowbytes = unsigned(3 * n * sizeof(T));
  if (lane == 0) {
    fence_proxy_async();
    mbar_expect_tx(bar, rowbytes * rows);
  }
  __syncwarp();
  for (int r = lane; r < rows; r += 32) {
    int y = (y0 - 1 + r) % n;
    if (y < 0) y += n;
    tma_row(buf + r * 3 * n, in + (size_t(pz) * n + y) * size_t(3 * n), rowbytes, bar);
  }
}

template <typename T>
__device__ __forceinline__ void tma_plane(T* buf, const T* in, int pz, int y0, int rows, int n, uint64_t* bar) {
  const unsigned rowbytes = unsigned(3 * n * sizeof(T));
  fence_proxy_async();
  mbar_expect_tx(bar, rowbytes * rows);
  for (int r = 0; r < rows; ++r) {
    int y = (y0 - 1 + r) % n;
    if (y < 0) y += n;
    tma_row(buf + r * 3 * n, in + (size_t(pz) * n + y) * size_t(3 * n), rowbytes, bar);
  }
}

StencilGeom stencil_geom_shape(int n, int ty, int zc, int stages, int occ) {
  StencilGeom g;
  g.occ = occ;
  g.ty = ty;
  g.ntiles = (n + ty - 1) / ty;
  g.zc = zc;
  g.nchunks = (n + zc - 1) / zc;
  g.stages = stages;
  return g;
}

StencilGeom stencil_geom(int n, int loads) {
  StencilGeom g;
  const int maxthreads = 512;
  int best_ty = 1;
  double best = 1e30;
  for (int ty = 1; ty <= n && n * (ty + 1) <= maxthreads; ++ty) {
    int tiles = (n + ty - 1) / ty;
    double waste = double(tiles) * (ty + 1) / n;
    if (waste < best - 1e-12) { best = waste; best_ty = ty; }
  }
  g.ty = best_ty;
  // tuning override (sweeps): PGJ_STENCIL_TY rows per tile, PGJ_STENCIL_ZC planes per chunk
  if (const char* e = std::getenv("PGJ_STENCIL_TY")) {
    const int v = std::atoi(e);
    if (v >= 1 && v <= n && n * (v + 1) <= maxthreads) g.ty = v;
  }
  g.ntiles = (n + g.ty - 1) / g.ty;
  // aim for >= ~2 blocks per SM across the launch, z chunks of at least 4 planes
  int want = (2 * 148 + loads * g.ntiles - 1) / (loads * g.ntiles);
  int maxchunks = n / 4 > 0 ? n / 4 : 1;
  int nch = want < 1 ? 1 : (want > maxchunks ? maxchunks : want);
  g.zc = (n + nch - 1) / nch;
  if (const char* e = std::getenv("PGJ_STENCIL_ZC")) {
    const int v = std::atoi(e);
    if (v >= 1 && v <= n) g.zc = v;
  }
  g.nchunks = (n + g.zc - 1) / g.zc;
  g.stages = 2;
  if (const char* e = std::getenv("PGJ_STENCIL_STAGES")) {
    const int v = std::atoi(e);
    if (v >= 2 && v <= kMaxPlaneStages) g.stages = v;
  }
  g.occ = 1;
  if (const char* e = std::getenv("PGJ_STENCIL_OCC")) g.occ = std::atoi(e) == 3 ? 3 : 1;
  return g;
}

template <typename T>
__device__ __forceinline__ void stage_plane(T* buf, const T* in, int pz, int y0, int rows, int n, int tid, int nthr) {
  const int rowlen = 3 * n;
  const int total = rows * rowlen;
  for (int i = tid; i < total; i += nthr) {
    const int row = i / rowlen;
    const int rem = i - row * rowlen;
    int y = (y0 - 1 + row) % n;
    if (y < 0) y += n;
    cp_async(buf + i, in + (size_t(pz) * n + y) * size_t(rowlen) + rem);
  }
  cp_commit();
}

// Three displacement components of one node or mode. FP32 keeps (x, y) as one packed pair, so an
// add or subtract of two triples is two instructions on sm_100 instead of three. A packed add
// rounds like a scalar one, but the compiler no longer fuses a preceding product into it (as it
// does in scalar code), so FP32 results differ from a scalar build in the last bits.
template <typename T>
struct Tri {
  T x, y, z;
  __device__ __forceinline__ T get(int c) const { return c == 0 ? x : (c == 1 ? y : z); }
  static __device__ __forceinline__ Tri make(T a, T b, T c) { return Tri{a, b, c}; }
  static __device__ __forceinline__ Tri load(const T* p) { return Tri{p[0], p[1], p[2]}; }
  __device__ __forceinline__ void store(T* p) const { p[0] = x; p[1] = y; p[2] = z; }
  friend __device__ __forceinline__ Tri operator+(Tri a, Tri b) { return Tri{a.x + b.x, a.y + b.y, a.z + b.z}; }
  friend __device__ __forceinline__ Tri operator-(Tri a, Tri b) { return Tri{a.x - b.x, a.y - b.y, a.z - b.z}; }
};
template <>
struct Tri<float> {
  float2 xy;
  float z;
  __device__ __forceinline__ float get(int c) const { return c == 0 ? xy.x : (c == 1 ? xy.y : z); }
  static __device__ __forceinline__ Tri make(float a, float b, float c) { return Tri{make_float2(a, b), c}; }
  static __device__ __forceinline__ Tri load(const float* p) { return Tri{make_float2(p[0], p[1]), p[2]}; }
  __device__ __forceinline__ void store(float* p) const { p[0] = xy.x; p[1] = xy.y; p[2] = z; }
  friend __device__ __forceinline__ Tri operator+(Tri a, Tri b) { return Tri{__fadd2_rn(a.xy, b.xy), a.z + b.z}; }
  friend __device__ __forceinline__ Tri operator-(Tri a, Tri b) {
    return Tri{__fadd2_rn(a.xy, make_float2(-b.xy.x, -b.xy.y)), a.z - b.z};
  }
};

// Read the 4 nodes of the face (x..x+1, row..row+1) from a staged plane ([row][x][component]) and
// form the face modes F[f], f = mx + 2 my: F[0] = sum, F[1] = x-difference, F[2] = y-difference,
// F[3] = both.
template <typename T>
__device__ __forceinline__ void face_modes(const T* buf, int row, int x, int n, Tri<T> (&F)[4], Tri<T>& own) {
  const int xp = (x + 1 == n) ? 0 : x + 1;
  const T* r0 = buf + row * 3 * n;
  const T* r1 = r0 + 3 * n;
  const Tri<T> u00 = Tri<T>::load(r0 + 3 * x), u10 = Tri<T>::load(r0 + 3 * xp);
  const Tri<T> u01 = Tri<T>::load(r1 + 3 * x), u11 = Tri<T>::load(r1 + 3 * xp);
  own = u00;
  const Tri<T> sx0 = u10 + u00, dx0 = u10 - u00, sx1 = u11 + u01, dx1 = u11 - u01;
  F[0] = sx1 + sx0;
  F[1] = dx1 + dx0;
  F[2] = sx1 - sx0;
  F[3] = dx1 - dx0;
}

// The same face modes one component at a time (the FP64 loop), in the compute type R (the staged
// values are of the storage type T: FP64, or FP32 for the FP64-arithmetic form of the FP32 operator).
template <typename T, typename R>
__device__ __forceinline__ void face_modes(const T* buf, int row, int x, int n, R (&F)[4][3], R (&own)[3]) {
  const int xp = (x + 1 == n) ? 0 : x + 1;
  const T* r0 = buf + row * 3 * n;
  const T* r1 = r0 + 3 * n;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const R u00 = R(r0[3 * x + c]), u10 = R(r0[3 * xp + c]), u01 = R(r1[3 * x + c]), u11 = R(r1[3 * xp + c]);
    own[c] = u00;
    const R sx0 = u10 + u00, dx0 = u10 - u00, sx1 = u11 + u01, dx1 = u11 - u01;
    F[0][c] = sx1 + sx0;
    F[1][c] = dx1 + dx0;
    F[2][c] = sx1 - sx0;
    F[3][c] = dx1 - dx0;
  }
}

// OCC = 1: blocks of up to 512 threads, registers unconstrained (128); OCC = 3: blocks of at most
// 256 threads, three resident per SM (85 registers). T is the storage type of p and q, R the
// arithmetic type (R = double with T = float: FP32 vectors, FP64 element actions and node sums, for
// high-contrast designs whose FP32 node sums cancel).
//
// PL: q of this launch is written component-planar, (3, N) per load (the FP32 recurrence vector of a
// slab-fused mixed context, read per component by the slab kernels); otherwise node-major with the
// components interleaved. p is read interleaved either way.
template <typename T, int MODE, int OCC, typename R = T, bool PL = false>
__global__ void __launch_bounds__(OCC == 1 ? 512 : 256, OCC) k_stencil(const StencilArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = A.n, TY = A.ty;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + n * ty, nthr = n * (TY + 1);
  const int load = blockIdx.z;
  const int nblk = gridDim.x * gridDim.y, blk = blockIdx.x + gridDim.x * blockIdx.y;
  const size_t N = size_t(n) * n * n;
  const int y0 = blockIdx.x * TY, z0 = blockIdx.y * A.zc;
  const int zc = min(A.zc, n - z0);
  const int ey = y0 - 1 + ty;
  const int eyw = (ey + n) % n;
  const bool out_row = (ty >= 1) && (ey < n);

  bool act = true;
  if (MODE == kPCG) act = A.scal[load].active != 0;
  else if (A.active_ext) act = A.active_ext[load] != 0;
  else if (MODE == kResidual && A.rel_flags) act = A.rel_flags[load].reliable != 0;
  // certification of a batched context: a design that took its last attempt keeps its certificate
  if (MODE == kResidual && A.scal[load].frozen) act = false;
  T* out = reinterpret_cast<T*>(A.out) + size_t(load) * 3 * N;
  if (!act) {
    if (MODE == kPlain && out_row) {
      for (int z = z0; z < z0 + zc; ++z) {
        const size_t node = (size_t(z) * n + ey) * n + tx;
        T* o = out + (PL ? node : 3 * node);
        o[0] = T(0); o[PL ? N : 1] = T(0); o[PL ? 2 * N : 2] = T(0);
      }
    }
    return;
  }
  const T* in = reinterpret_cast<const T*>(A.in) + size_t(load) * 3 * N;

  // plane j (node plane z0 - 1 + j) sits in buffer j % NS; with TMA staging every buffer is refilled
  // as soon as the block barrier after its last read has passed, so NS - 1 planes stay in flight
  const int NS = A.tma ? A.stages : 2;
  const int planevals = (TY + 2) * 3 * n;
  const int nt = n * (TY + 1);
  T* bufs = reinterpret_cast<T*>(smem_raw);
  // corner exchange in the arithmetic type, double-buffered by step parity:
  // [parity][corner 10 / 01 / 11][thread][3] (n is even, so the plane buffers end 8-byte aligned)
  R* xch = reinterpret_cast<R*>(bufs + NS * planevals);
  const int xsz = 3 * nt * 3;
  double* red = reinterpret_cast<double*>(xch + 2 * xsz + 2);  // 32 * 4, 16-byte padded
  red = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(red) + 15) & ~uintptr_t(15));
  uint64_t* bars = reinterpret_cast<uint64_t*>(red + 32 * 4);  // NS mbarriers (TMA staging)
  const bool tma = A.tma != 0;
  const int nplanes = zc + 2;

  // prologue: planes j = 0 .. NS-1 (plane 0 is z0 - 1); plane 0 gives the first lower face
  bool bad = false;
  if (tma) {
    if (tid == 0) {
      for (int b = 0; b < NS; ++b) mbar_init(&bars[b], 1);
      fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0)
      for (int j = 0; j < NS && j < nplanes; ++j)
        tma_plane(bufs + j * planevals, in, (z0 - 1 + j + n) % n, y0, TY + 2, n, &bars[j]);
    bad = !mbar_wait(&bars[0], 0);  // every thread observes the arrival (acquire)
  } else {
    stage_plane(bufs, in, (z0 - 1 + n) % n, y0, TY + 2, n, tid, nthr);
    stage_plane(bufs + planevals, in, z0 % n, y0, TY + 2, n, tid, nthr);
    cp_wait_one();
    __syncthreads();
  }
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  if constexpr (sizeof(R) == 4) {
    // FP32: packed-pair arithmetic (Tri) and two z-steps per loop trip, which removes the copies of
    // the carried face modes; 47 vs 51 us at n = 64, 6 loads. FP64 keeps the one-step form below:
    // the same restructuring made it slower (64 vs 61 us). One block barrier per step: sharing one
    // barrier between the two steps of a trip (four exchange slots) halved the barrier stalls but
    // measured 2 us slower (46.1 vs 43.7 us), with the own node values of two planes live.
    // lower-face modes, upper-plane carry and own node value of the plane below, in two sets that
    // swap roles every z-step (no copies at the loop edge)
    Tri<T> FA[4], UA[4], ownA, FB[4], UB[4], ownB;
    face_modes(bufs, ty, tx, n, FA, ownB);
    if (tma) {
      // buffer 0 is free once every thread has read plane 0
      if (__syncthreads_or(bad)) {
        if (tid == 0 && A.err) atomicExch(A.err, 1);
        return;
      }
      if (tid == 0 && NS < nplanes) tma_plane(bufs, in, (z0 - 1 + NS) % n, y0, TY + 2, n, &bars[0]);
    }
#pragma unroll
    for (int f = 0; f < 4; ++f) UA[f] = Tri<T>::make(T(0), T(0), T(0));
    ownA = Tri<T>::make(T(0), T(0), T(0));

    const double* aa = A.a + size_t(load / A.lpd) * N;  // this load's design

    // element densities are read one plane ahead so their latency overlaps the previous plane
    const double* arow = aa + size_t(eyw) * n + tx;
    const size_t aplane = size_t(n) * n;
    int za = (z0 - 1 + n) % n;  // element plane of the next density read (wraps incrementally)
    double a_next = __ldg(arow + size_t(za) * aplane);
    // buffer / phase bookkeeping without divisions: plane j = s + 1 sits in buffer jb with mbarrier
    // parity jpar; after the step's barrier that buffer takes plane s + 1 + NS (node plane zr)
    int jb = 1 % NS;
    unsigned jpar = 0u;
    int zr = (z0 + NS) % n;
    const bool full_warp0 = nthr >= 32;
    const int tl = ty * n + (tx == 0 ? n - 1 : tx - 1);          // element to the left (periodic x)
    const int tb = (ty >= 1 ? ty - 1 : 0) * n + tx;              // element below
    const int tbl = (ty >= 1 ? ty - 1 : 0) * n + (tx == 0 ? n - 1 : tx - 1);
    const int tme = ty * n + tx;

    // One element plane s: F0 / Up / own0 hold the lower face modes, the carry from the element
    // below and the own node value of node plane ez; F1 / U / own1 receive those of the next plane.
    // Returns false when a bounded wait gave up (the block then leaves).
    auto step = [&](int s, const Tri<T> (&F0)[4], const Tri<T> (&Up)[4], const Tri<T>& own0, Tri<T> (&F1)[4],
                    Tri<T> (&U)[4], Tri<T>& own1) -> bool {
      const int ez = z0 - 1 + s;           // element plane
      const T ae = T(a_next);
      if (s < zc) {
        za = za + 1 == n ? 0 : za + 1;
        a_next = __ldg(arow + size_t(za) * aplane);
      }
      T* cur = bufs + jb * planevals;
      if (tma) {
        bad = bad || !mbar_wait(&bars[jb], jpar);
      } else {
        cp_wait_all();
        __syncthreads();
        if (s < zc) stage_plane(((s & 1) ? bufs + planevals : bufs), in, (z0 + s + 1) % n, y0, TY + 2, n, tid, nthr);
      }

      face_modes(cur, ty, tx, n, F1, own1);
      // element modes: z level
      T Q[8][3];
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        const Tri<T> sum = F1[f] + F0[f], dif = F1[f] - F0[f];
#pragma unroll
        for (int c = 0; c < 3; ++c) { Q[f][c] = sum.get(c); Q[f + 4][c] = dif.get(c); }
      }
      T P[8][3];
      element_modal<T>(Q, ae, A.kc, P);
      // z-level transpose: U -> upper plane (ez+1), G -> lower plane (ez)
      Tri<T> G[4];
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        const Tri<T> lo = Tri<T>::make(P[f][0], P[f][1], P[f][2]);
        const Tri<T> hi = Tri<T>::make(P[f + 4][0], P[f + 4][1], P[f + 4][2]);
        U[f] = lo + hi;
        G[f] = (lo - hi) + Up[f];
      }
      // lower face of the element (node plane ez) as its four corner nodes: this thread keeps the
      // (x, y) corner and hands (x+1, y), (x, y+1), (x+1, y+1) to their owners through shared memory
      Tri<T> c00;
      T* xb = xch + (s & 1) * xsz;
      if (s >= 1) {
        const Tri<T> ly0 = G[0] - G[2], ly1 = G[1] - G[3];
        const Tri<T> uy0 = G[0] + G[2], uy1 = G[1] + G[3];
        c00 = ly0 - ly1;
        (ly0 + ly1).store(xb + (0 * nt + tme) * 3);
        (uy0 - uy1).store(xb + (1 * nt + tme) * 3);
        (uy0 + uy1).store(xb + (2 * nt + tme) * 3);
      }
      // one barrier per step: corners published, plane jb fully read, timeouts agreed on
      if (__syncthreads_or(bad)) {
        if (tid == 0 && A.err) atomicExch(A.err, 1);
        return false;
      }
      if (tma && s + 1 + NS < nplanes) {
        // warp 0 refills (its lanes issue the rows in parallel); a block of fewer than 32 threads
        // has no full warp, and thread 0 issues the rows alone
        if (full_warp0) {
          if (tid < 32) tma_plane_warp(cur, in, zr, y0, TY + 2, n, &bars[jb], tid);
        } else if (tid == 0) {
          tma_plane(cur, in, zr, y0, TY + 2, n, &bars[jb]);
        }
      }
      if (++jb == NS) { jb = 0; jpar ^= 1u; }
      zr = zr + 1 == n ? 0 : zr + 1;
      if (s >= 1 && out_row) {
        const Tri<T> qx = ((c00 + Tri<T>::load(xb + (0 * nt + tl) * 3)) + Tri<T>::load(xb + (1 * nt + tb) * 3)) +
                          Tri<T>::load(xb + (2 * nt + tbl) * 3);
        const size_t node = (size_t(ez) * n + ey) * n + tx;
        T* o = out + (PL ? node : 3 * node);
        // FP32 never runs the residual mode (the host rejects it); the branch is kept because the
        // build without it allocates registers differently and measured 0.6 us slower
        if (MODE == kResidual) {
          const double* fl = A.f + size_t(load) * 3 * N + 3 * node;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const double rv = fl[c] - double(qx.get(c));
            o[c] = T(rv);
            acc[0] += rv * rv;
            acc[1 + c] += rv;
          }
        } else {
          if constexpr (PL) {
            o[0] = qx.get(0); o[N] = qx.get(1); o[2 * N] = qx.get(2);
          } else {
            qx.store(o);
          }
          if (MODE == kPCG) {
#pragma unroll
            for (int c = 0; c < 3; ++c) acc[0] += double(own0.get(c)) * double(qx.get(c));
          }
        }
      }
      return true;
    };
    // two steps per trip with the sets swapped (the carries stay where they were written)
    for (int s = 0; s <= zc; s += 2) {
      if (!step(s, FA, UA, ownA, FB, UB, ownB)) return;
      if (s + 1 > zc) break;
      if (!step(s + 1, FB, UB, ownB, FA, UA, ownA)) return;
    }
  } else {
    R F0[4][3], own[3], dummy[3];
    face_modes(bufs, ty, tx, n, F0, dummy);
    if (tma) {
      // buffer 0 is free once every thread has read plane 0
      if (__syncthreads_or(bad)) {
        if (tid == 0 && A.err) atomicExch(A.err, 1);
        return;
      }
      if (tid == 0 && NS < nplanes) tma_plane(bufs, in, (z0 - 1 + NS) % n, y0, TY + 2, n, &bars[0]);
    }
    R Up[4][3];
#pragma unroll
    for (int f = 0; f < 4; ++f)
#pragma unroll
      for (int c = 0; c < 3; ++c) Up[f][c] = R(0);
#pragma unroll
    for (int c = 0; c < 3; ++c) own[c] = R(0);

    const double* aa = A.a + size_t(load / A.lpd) * N;  // this load's design

    // element densities are read one plane ahead so their latency overlaps the previous plane
    const double* arow = aa + size_t(eyw) * n + tx;
    const size_t aplane = size_t(n) * n;
    int za = (z0 - 1 + n) % n;  // element plane of the next density read (wraps incrementally)
    double a_next = __ldg(arow + size_t(za) * aplane);
    // buffer / phase bookkeeping without divisions: plane j = s + 1 sits in buffer jb with mbarrier
    // parity jpar; after the step's barrier that buffer takes plane s + 1 + NS (node plane zr)
    int jb = 1 % NS;
    unsigned jpar = 0u;
    int zr = (z0 + NS) % n;
    const bool full_warp0 = nthr >= 32;
    const int tl = ty * n + (tx == 0 ? n - 1 : tx - 1);          // element to the left (periodic x)
    const int tb = (ty >= 1 ? ty - 1 : 0) * n + tx;              // element below
    const int tbl = (ty >= 1 ? ty - 1 : 0) * n + (tx == 0 ? n - 1 : tx - 1);
    const int tme = ty * n + tx;
    for (int s = 0; s <= zc; ++s) {
      const int ez = z0 - 1 + s;           // element plane
      const R ae = R(a_next);
      if (s < zc) {
        za = za + 1 == n ? 0 : za + 1;
        a_next = __ldg(arow + size_t(za) * aplane);
      }
      T* cur = bufs + jb * planevals;
      if (tma) {
        bad = bad || !mbar_wait(&bars[jb], jpar);
      } else {
        cp_wait_all();
        __syncthreads();
        if (s < zc) stage_plane(((s & 1) ? bufs + planevals : bufs), in, (z0 + s + 1) % n, y0, TY + 2, n, tid, nthr);
      }

      R F1[4][3], own1[3];
      face_modes(cur, ty, tx, n, F1, own1);
      // element modes: z level
      R Q[8][3];
#pragma unroll
      for (int f = 0; f < 4; ++f)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          Q[f][c] = F1[f][c] + F0[f][c];
          Q[f + 4][c] = F1[f][c] - F0[f][c];
        }
      R P[8][3];
      element_modal<R>(Q, ae, A.kc, P);
      // z-level transpose: U -> upper plane (ez+1), G -> lower plane (ez)
      R U[4][3], G[4][3];
#pragma unroll
      for (int f = 0; f < 4; ++f)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          U[f][c] = P[f][c] + P[f + 4][c];
          G[f][c] = (P[f][c] - P[f + 4][c]) + Up[f][c];
        }
      // lower face of the element (node plane ez) as its four corner nodes: this thread keeps the
      // (x, y) corner and hands (x+1, y), (x, y+1), (x+1, y+1) to their owners through shared memory
      R c00[3];
      R* xb = xch + (s & 1) * xsz;
      if (s >= 1) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const R ly0 = G[0][c] - G[2][c], ly1 = G[1][c] - G[3][c];
          const R uy0 = G[0][c] + G[2][c], uy1 = G[1][c] + G[3][c];
          c00[c] = ly0 - ly1;
          xb[(0 * nt + tme) * 3 + c] = ly0 + ly1;
          xb[(1 * nt + tme) * 3 + c] = uy0 - uy1;
          xb[(2 * nt + tme) * 3 + c] = uy0 + uy1;
        }
      }
      // one barrier per step: corners published, plane jb fully read, timeouts agreed on
      if (__syncthreads_or(bad)) {
        if (tid == 0 && A.err) atomicExch(A.err, 1);
        return;
      }
      if (tma && s + 1 + NS < nplanes) {
        // warp 0 refills (its lanes issue the rows in parallel); a block of fewer than 32 threads
        // has no full warp, and thread 0 issues the rows alone
        if (full_warp0) {
          if (tid < 32) tma_plane_warp(cur, in, zr, y0, TY + 2, n, &bars[jb], tid);
        } else if (tid == 0) {
          tma_plane(cur, in, zr, y0, TY + 2, n, &bars[jb]);
        }
      }
      if (++jb == NS) { jb = 0; jpar ^= 1u; }
      zr = zr + 1 == n ? 0 : zr + 1;
      if (s >= 1 && out_row) {
        R qx[3];
#pragma unroll
        for (int c = 0; c < 3; ++c)
          qx[c] = ((c00[c] + xb[(0 * nt + tl) * 3 + c]) + xb[(1 * nt + tb) * 3 + c]) + xb[(2 * nt + tbl) * 3 + c];
        const size_t node = (size_t(ez) * n + ey) * n + tx;
        T* o = out + (PL ? node : 3 * node);
        if (MODE == kResidual) {
          const double* fl = A.f + size_t(load) * 3 * N + 3 * node;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const double rv = fl[c] - double(qx[c]);
            o[c] = T(rv);
            acc[0] += rv * rv;
            acc[1 + c] += rv;
          }
        } else {
#pragma unroll
          for (int c = 0; c < 3; ++c) o[PL ? c * N : c] = T(qx[c]);
          if (MODE == kPCG) {
#pragma unroll
            for (int c = 0; c < 3; ++c) acc[0] += double(own[c]) * double(qx[c]);
          }
        }
      }
#pragma unroll
      for (int f = 0; f < 4; ++f)
#pragma unroll
        for (int c = 0; c < 3; ++c) { F0[f][c] = F1[f][c]; Up[f][c] = U[f][c]; }
#pragma unroll
      for (int c = 0; c < 3; ++c) own[c] = own1[c];
    }

  }

  if (MODE == kPlain) return;
  block_sum<4>(acc, red);
  double* part = A.partials + size_t(load) * kPartialQ * kMaxPartials;
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < 4; ++k) part[k * kMaxPartials + blk] = acc[k];
  }
  LoadScalars& S = A.scal[load];
  if (!last_block(&S.ticket[kTicketApply], nblk)) return;
  if (tid < 32) {
    if (MODE == kPCG) {
      const double den = warp_sum_partials(part, nblk);
      if (tid == 0) {
        const double rz = S.rz;
        const bool valid = isfinite(den) && den > 0.0 && isfinite(rz) && rz > 0.0;
        S.failed = valid ? 0 : 1;
        S.alpha = valid ? rz / den : 0.0;
      }
    } else {
      double v[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) v[k] = warp_sum_partials(part + k * kMaxPartials, nblk);
      if (tid == 0) {
        S.res2 = v[0];
        S.absolute = sqrt(v[0]);
        const double inv = 1.0 / double(N);
#pragma unroll
        for (int c = 0; c < 3; ++c) S.mean_r[c] = v[1 + c] * inv;
      }
    }
  }
}

// ------------------------------------------------------------------ halo-free recurrence operator
// The FP32 recurrence operator of slab-fused mixed contexts, without the halo element row of
// k_stencil: a block owns TY node rows (TY divides n) and exactly the TY element rows whose lower
// node row is one of them, so no element is computed twice. Thread (x, ty) owns element (x, y0 + ty).
// A node row y0 + ty, ty >= 1, gets all four corner contributions inside the block (same order as
// k_stencil) and is stored. The first row y0 of a tile gets its own elements' corners here; those of
// the element row below the tile are the upper corners of the top element row of the tile below, which
// that block writes, per z-plane and tile, to the boundary array qb ([load][z][tile][component][x]);
// the slab update (k_fxy) adds qb to q on the rows y % TY == 0 as it reads q. (Adding the two parts
// atomically onto zeroed rows of q instead measured slower: the atomics cost the operator 4.6 us and
// re-zeroing the rows cost the slab update 4 us.) p^T q counts each part in the block that computes
// it, with p of the node it belongs to (the upper face of the top row), so alpha = r.z / p^T q is the
// quantity of the halo form; only the rounding of the first rows differs.
// Planes are staged as TY + 1 node rows (y0 .. y0 + TY), q is written component-planar, p is read
// interleaved.
__device__ __forceinline__ void face_modes_top(const float* buf, int row, int x, int n, Tri<float> (&F)[4],
                                               Tri<float>& own, Tri<float>& top) {
  const int xp = (x + 1 == n) ? 0 : x + 1;
  const float* r0 = buf + row * 3 * n;
  const float* r1 = r0 + 3 * n;
  const Tri<float> u00 = Tri<float>::load(r0 + 3 * x), u10 = Tri<float>::load(r0 + 3 * xp);
  const Tri<float> u01 = Tri<float>::load(r1 + 3 * x), u11 = Tri<float>::load(r1 + 3 * xp);
  own = u00;
  top = u01;
  const Tri<float> sx0 = u10 + u00, dx0 = u10 - u00, sx1 = u11 + u01, dx1 = u11 - u01;
  F[0] = sx1 + sx0;
  F[1] = dx1 + dx0;
  F[2] = sx1 - sx0;
  F[3] = dx1 - dx0;
}

__global__ void __launch_bounds__(256, 2) k_stencil_hf(const StencilArgs A) {
  using T = float;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = A.n, TY = A.ty;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + n * ty, nthr = n * TY;
  const int load = blockIdx.z;
  const int ntiles = gridDim.x;
  const int nblk = gridDim.x * gridDim.y, blk = blockIdx.x + gridDim.x * blockIdx.y;
  const size_t N = size_t(n) * n * n;
  const int y0 = blockIdx.x * TY, z0 = blockIdx.y * A.zc;
  const int zc = min(A.zc, n - z0);
  const int ey = y0 + ty;  // element row = own node row (< n: TY divides n)
  LoadScalars& S = A.scal[load];
  if (S.active == 0) return;
  T* out = reinterpret_cast<T*>(A.out) + size_t(load) * 3 * N;
  // boundary rows for the tile above (the first row of tile blockIdx.x + 1, periodic in y)
  T* qb = reinterpret_cast<T*>(A.qb) + size_t(load) * n * ntiles * 3 * n +
          size_t(blockIdx.x + 1 == ntiles ? 0 : blockIdx.x + 1) * 3 * n + tx;
  const T* in = reinterpret_cast<const T*>(A.in) + size_t(load) * 3 * N;

  const int NS = A.tma ? A.stages : 2;
  const int rows = TY + 1;
  const int planevals = rows * 3 * n;
  const int nt = n * TY;
  T* bufs = reinterpret_cast<T*>(smem_raw);
  T* xch = bufs + NS * planevals;  // [parity][corner 10 / 01 / 11][thread][3]
  const int xsz = 3 * nt * 3;
  double* red = reinterpret_cast<double*>(xch + 2 * xsz + 2);
  red = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(red) + 15) & ~uintptr_t(15));
  uint64_t* bars = reinterpret_cast<uint64_t*>(red + 32 * 4);
  const bool tma = A.tma != 0;
  const int nplanes = zc + 2;
  // the staging helpers take rows (y0' - 1 + r) mod n: y0' = y0 + 1 gives rows y0 .. y0 + TY
  const int ys = y0 + 1;

  bool bad = false;
  if (tma) {
    if (tid == 0) {
      for (int b = 0; b < NS; ++b) mbar_init(&bars[b], 1);
      fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0)
      for (int j = 0; j < NS && j < nplanes; ++j)
        tma_plane(bufs + j * planevals, in, (z0 - 1 + j + n) % n, ys, rows, n, &bars[j]);
    bad = !mbar_wait(&bars[0], 0);
  } else {
    stage_plane(bufs, in, (z0 - 1 + n) % n, ys, rows, n, tid, nthr);
    stage_plane(bufs + planevals, in, z0 % n, ys, rows, n, tid, nthr);
    cp_wait_one();
    __syncthreads();
  }
  double acc = 0.0;
  Tri<T> FA[4], UA[4], ownA, topA, FB[4], UB[4], ownB, topB;
  face_modes_top(bufs, ty, tx, n, FA, ownB, topB);
  if (tma) {
    if (__syncthreads_or(bad)) {
      if (tid == 0 && A.err) atomicExch(A.err, 1);
      return;
    }
    if (tid == 0 && NS < nplanes) tma_plane(bufs, in, (z0 - 1 + NS) % n, ys, rows, n, &bars[0]);
  }
#pragma unroll
  for (int f = 0; f < 4; ++f) UA[f] = Tri<T>::make(T(0), T(0), T(0));
  ownA = Tri<T>::make(T(0), T(0), T(0));
  topA = ownA;

  const double* arow = A.a + size_t(load / A.lpd) * N + size_t(ey) * n + tx;
  const size_t aplane = size_t(n) * n;
  int za = (z0 - 1 + n) % n;
  double a_next = __ldg(arow + size_t(za) * aplane);
  int jb = 1 % NS;
  unsigned jpar = 0u;
  int zr = (z0 + NS) % n;
  const bool full_warp0 = nthr >= 32;
  const int txl = tx == 0 ? n - 1 : tx - 1;
  const int tl = ty * n + txl;                       // element to the left (periodic x)
  const int tb = (ty >= 1 ? ty - 1 : 0) * n + tx;    // element below (inside the tile)
  const int tbl = (ty >= 1 ? ty - 1 : 0) * n + txl;
  const int tme = ty * n + tx;
  const bool top_row = ty == TY - 1;

  auto step = [&](int s, const Tri<T> (&F0)[4], const Tri<T> (&Up)[4], const Tri<T>& own0, const Tri<T>& top0,
                  Tri<T> (&F1)[4], Tri<T> (&U)[4], Tri<T>& own1, Tri<T>& top1) -> bool {
    const int ez = z0 - 1 + s;
    const T ae = T(a_next);
    if (s < zc) {
      za = za + 1 == n ? 0 : za + 1;
      a_next = __ldg(arow + size_t(za) * aplane);
    }
    T* cur = bufs + jb * planevals;
    if (tma) {
      bad = bad || !mbar_wait(&bars[jb], jpar);
    } else {
      cp_wait_all();
      __syncthreads();
      if (s < zc) stage_plane(((s & 1) ? bufs + planevals : bufs), in, (z0 + s + 1) % n, ys, rows, n, tid, nthr);
    }
    face_modes_top(cur, ty, tx, n, F1, own1, top1);
    T Q[8][3];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      const Tri<T> sum = F1[f] + F0[f], dif = F1[f] - F0[f];
#pragma unroll
      for (int c = 0; c < 3; ++c) { Q[f][c] = sum.get(c); Q[f + 4][c] = dif.get(c); }
    }
    T P[8][3];
    element_modal<T>(Q, ae, A.kc, P);
    Tri<T> G[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      const Tri<T> lo = Tri<T>::make(P[f][0], P[f][1], P[f][2]);
      const Tri<T> hi = Tri<T>::make(P[f + 4][0], P[f + 4][1], P[f + 4][2]);
      U[f] = lo + hi;
      G[f] = (lo - hi) + Up[f];
    }
    Tri<T> c00, c01;
    T* xb = xch + (s & 1) * xsz;
    if (s >= 1) {
      const Tri<T> ly0 = G[0] - G[2], ly1 = G[1] - G[3];
      const Tri<T> uy0 = G[0] + G[2], uy1 = G[1] + G[3];
      c00 = ly0 - ly1;
      c01 = uy0 - uy1;
      (ly0 + ly1).store(xb + (0 * nt + tme) * 3);
      c01.store(xb + (1 * nt + tme) * 3);
      (uy0 + uy1).store(xb + (2 * nt + tme) * 3);
    }
    if (__syncthreads_or(bad)) {
      if (tid == 0 && A.err) atomicExch(A.err, 1);
      return false;
    }
    if (tma && s + 1 + NS < nplanes) {
      if (full_warp0) {
        if (tid < 32) tma_plane_warp(cur, in, zr, ys, rows, n, &bars[jb], tid);
      } else if (tid == 0) {
        tma_plane(cur, in, zr, ys, rows, n, &bars[jb]);
      }
    }
    if (++jb == NS) { jb = 0; jpar ^= 1u; }
    zr = zr + 1 == n ? 0 : zr + 1;
    if (s >= 1) {
      Tri<T> qx = c00 + Tri<T>::load(xb + (0 * nt + tl) * 3);
      if (ty >= 1) qx = (qx + Tri<T>::load(xb + (1 * nt + tb) * 3)) + Tri<T>::load(xb + (2 * nt + tbl) * 3);
      const size_t node = (size_t(ez) * n + ey) * n + tx;
      T* o = out + node;
      o[0] = qx.get(0); o[N] = qx.get(1); o[2 * N] = qx.get(2);
#pragma unroll
      for (int c = 0; c < 3; ++c) acc += double(own0.get(c)) * double(qx.get(c));
      if (top_row) {
        // node (x, y0 + TY) of plane ez: this element's (x, y+1) corner and the left element's (x+1, y+1)
        const Tri<T> bq = c01 + Tri<T>::load(xb + (2 * nt + tl) * 3);
        T* b = qb + size_t(ez) * ntiles * 3 * n;
        b[0] = bq.get(0); b[n] = bq.get(1); b[2 * n] = bq.get(2);
#pragma unroll
        for (int c = 0; c < 3; ++c) acc += double(top0.get(c)) * double(bq.get(c));
      }
    }
    return true;
  };
  for (int s = 0; s <= zc; s += 2) {
    if (!step(s, FA, UA, ownA, topA, FB, UB, ownB, topB)) return;
    if (s + 1 > zc) break;
    if (!step(s + 1, FB, UB, ownB, topB, FA, UA, ownA, topA)) return;
  }

  double v1[1] = {acc};
  block_sum<1>(v1, red);
  double* part = A.partials + size_t(load) * kPartialQ * kMaxPartials;
  if (tid == 0) part[blk] = v1[0];
  if (!last_block(&S.ticket[kTicketApply], nblk)) return;
  if (tid < 32) {
    const double den = warp_sum_partials(part, nblk);
    if (tid == 0) {
      const double rz = S.rz;
      const bool valid = isfinite(den) && den > 0.0 && isfinite(rz) && rz > 0.0;
      S.failed = valid ? 0 : 1;
      S.alpha = valid ? rz / den : 0.0;
    }
  }
}

// Halo-free geometry for grid edge n and `lpd` loads per design: TY the largest divisor of n with
// n TY <= 256 threads (TY >= 2), and the z chunking that fills the launch's block slots best
// (blocks per design over whole waves of 148 SMs times the blocks per SM, times the share of element
// planes that are not recomputed at chunk starts). Depends on n and lpd only, so a design's
// decomposition (and summation order) is the same alone and in a batch. PGJ_HF_TY / PGJ_HF_ZC pin it.
StencilGeom hf_geom(int n, int lpd) {
  StencilGeom g;
  g.ty = 2;
  for (int t = 2; t <= n && n * t <= 256; ++t)
    if (n % t == 0) g.ty = t;
  if (const char* e = std::getenv("PGJ_HF_TY")) {
    const int v = std::atoi(e);
    if (v >= 2 && v <= n && n % v == 0 && n * v <= 256) g.ty = v;
  }
  g.ntiles = n / g.ty;
  const int threads = n * g.ty;
  int bps = 65536 / (threads * 128);
  bps = bps < 1 ? 1 : (bps > 8 ? 8 : bps);
  const int slots = 148 * bps;
  double best = -1.0;
  int best_zc = n;
  for (int nch = 1; nch <= (n / 4 > 1 ? n / 4 : 1); ++nch) {
    const int zc = (n + nch - 1) / nch;
    const int chunks = (n + zc - 1) / zc;
    const long blocks = long(lpd) * g.ntiles * chunks;
    const long waves = (blocks + slots - 1) / slots;
    const double eff = double(blocks) / double(waves * slots) * double(zc) / double(zc + 1);
    if (eff > best + 1e-9) { best = eff; best_zc = zc; }
  }
  g.zc = best_zc;
  if (const char* e = std::getenv("PGJ_HF_ZC")) {
    const int v = std::atoi(e);
    if (v >= 1 && v <= n) g.zc = v;
  }
  g.nchunks = (n + g.zc - 1) / g.zc;
  g.stages = 2;
  g.occ = 1;
  return g;
}

int launch_recurrence_operator(pgj_ctx* c, int loads, int prec, cudaStream_t s) {
  if (uses_hf(c, prec)) return launch_stencil_hf(c, loads, s);
  return launch_stencil(c, kPCG, loads, prec, c->p, c->q, nullptr, nullptr, s);
}

int launch_stencil_hf(pgj_ctx* c, int loads, cudaStream_t s) {
  const int n = c->n;
  const StencilGeom& g = c->hg;
  StencilArgs A;
  A.n = n; A.ty = g.ty; A.zc = g.zc;
  A.lpd = c->lpd;
  A.a = c->a; A.in = c->p; A.out = c->q; A.f = nullptr; A.active_ext = nullptr;
  A.scal = c->scal; A.partials = c->partials; A.kc = c->kc; A.iteration_cap = c->cap;
  A.err = c->cond + 2;
  A.rel_flags = nullptr;
  A.qb = c->qb;
  const size_t rowb = 3 * size_t(n) * sizeof(float);
  A.tma = (rowb % 16 == 0) && (reinterpret_cast<uintptr_t>(c->p) % 16 == 0) ? 1 : 0;
  A.stages = A.tma ? g.stages : 2;
  if (g.ntiles * g.nchunks > kMaxPartials || n * g.ty > 256) return PGJ_ERR_UNSUPPORTED;
  const size_t smem = sizeof(float) * size_t(A.stages) * (g.ty + 1) * 3 * n + sizeof(float) * 2 * 9 * g.ty * n +
                      32 * 4 * 8 + 16 + 8 * A.stages + 64;
  k_stencil_hf<<<dim3(g.ntiles, g.nchunks, loads), dim3(n, g.ty), smem, s>>>(A);
  return check_launch();
}

// Tile table: shapes per (grid edge, precision) picked offline by the project's tuner
// (partial-green-jacobi_b200/tune_tiles.py, which times every candidate on a B200 and writes
// pgj_tiles.inc). Contexts of a tabulated size take these shapes without timing anything, so the
// block decomposition, and with it the summation order of every block-partial reduction, is the
// same in every process, batch size and run. Sizes outside the table are tuned by timing at
// context creation (below); PGJ_AUTOTUNE=1 forces timing for every size (that is how the table is
// made).
static const TileEntry kTileTable[] = {
#include "pgj_tiles.inc"
    {0, 0, 0, 0, 0, 0, 0, 0, 0}};

bool tile_table(int n, int prec, TileEntry* out) {
  if (const char* e = std::getenv("PGJ_AUTOTUNE"))
    if (e[0] == '1') return false;
  for (const TileEntry& t : kTileTable)
    if (t.n == n && t.prec == prec) { *out = t; return true; }
  return false;
}

// Tile autotuner: times the operator (the loads of one design, plain mode) for candidate tile shapes
// on the context's own buffers and keeps the fastest. Results are cached per (n, loads per design,
// precision) for the process, so contexts created later, batched ones included, reuse the choice
// (and with it the order of the operator's block partial sums).
static std::mutex g_tune_mutex;
static std::map<std::tuple<int, int, int>, StencilGeom> g_tuned;

int autotune_stencil(pgj_ctx* c, cudaStream_t s) {
  const int n = c->n;
  const auto key = std::make_tuple(n, c->lpd, c->prec);
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) {
      c->sg = it->second;
      TileEntry t;
      c->tile_source = tile_table(n, c->prec, &t) ? 1 : 0;
      return PGJ_OK;
    }
  }
  if (std::getenv("PGJ_STENCIL_TY") || std::getenv("PGJ_STENCIL_ZC") || std::getenv("PGJ_STENCIL_OCC")) {
    c->tile_source = 2;
    return PGJ_OK;  // manual override
  }
  TileEntry t;
  if (tile_table(n, c->prec, &t)) {
    c->sg = stencil_geom_shape(n, t.ty, t.zc, t.stages, t.occ);
    c->tile_source = 1;
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tuned[key] = c->sg;
    return PGJ_OK;
  }
  c->tile_source = 0;
  std::vector<int> tys;
  for (int ty : {1, 2, 3, 4, 5, 6, 7, 8, 12, 16, 31})
    if (ty <= n && n * (ty + 1) <= 512 && (ty + 1) * n >= 32) tys.push_back(ty);
  if (tys.empty()) tys.push_back(c->sg.ty);
  std::vector<int> zcs;
  for (int zc : {4, 8, 16, 32})
    if (zc <= n) zcs.push_back(zc);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  StencilGeom best = c->sg;
  float best_ms = 1e30f;
  const void* in = c->p;
  void* out = c->q;
  // bring the clocks up before timing anything
  for (int r = 0; r < 30; ++r) launch_stencil(c, kPlain, c->lpd, c->prec, in, out, nullptr, nullptr, s, nullptr, true);
  for (int ty : tys)
    for (int zc : zcs)
      for (int occ : {1, 3})
      for (int stages = 2; stages <= kMaxPlaneStages; stages += 2) {
        if (occ == 3 && n * (ty + 1) > 256) continue;
        StencilGeom g = stencil_geom_shape(n, ty, zc, stages, occ);
        if (g.ntiles * g.nchunks > kMaxPartials) continue;
        c->sg = g;
        int st = launch_stencil(c, kPlain, c->lpd, c->prec, in, out, nullptr, nullptr, s, nullptr, true);  // warm
        if (st) { cudaEventDestroy(e0); cudaEventDestroy(e1); return st; }
        float ms = 1e30f;
        for (int trial = 0; trial < 2; ++trial) {  // best of two trials of five launches
          cudaEventRecord(e0, s);
          for (int r = 0; r < 5; ++r) launch_stencil(c, kPlain, c->lpd, c->prec, in, out, nullptr, nullptr, s, nullptr, true);
          cudaEventRecord(e1, s);
          cudaEventSynchronize(e1);
          float t = 0.f;
          cudaEventElapsedTime(&t, e0, e1);
          ms = t < ms ? t : ms;
        }
        if (ms < best_ms) { best_ms = ms; best = g; }
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->sg = best;
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  g_tuned[key] = best;
  return check_launch();
}

// Self-test of the bounded device wait: an mbarrier armed for 16 bytes that no copy will deliver;
// the wait must give up after `tries` polls and report it. No asynchronous copy is ever issued.
__global__ void k_wait_selftest(int tries, int* flag) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_expect_tx(&bar, 16);  // the transaction count never drains
  const bool ok = mbar_wait(&bar, 0, tries);
  if (__syncthreads_or(!ok) && threadIdx.x == 0) *flag = 1;
}

int launch_wait_selftest(int tries, int* flag, cudaStream_t s) {
  k_wait_selftest<<<1, 32, 0, s>>>(tries, flag);
  return check_launch();
}

template <int OCC>
static void set_stencil_smem(int lim) {
  cudaFuncSetAttribute(k_stencil<float, kPlain, OCC>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_stencil<float, kPCG, OCC>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_stencil<double, kPlain, OCC>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_stencil<double, kPCG, OCC>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_stencil<double, kResidual, OCC>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_stencil<float, kPCG, OCC, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_stencil<float, kPCG, OCC, float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_stencil<float, kPlain, OCC, float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_stencil<float, kPCG, OCC, double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
}

int prepare_stencil_kernels() {
  set_stencil_smem<1>(220 * 1024);  // below the 227 KB opt-in less the static shared memory
  set_stencil_smem<3>(72 * 1024);
  cudaFuncSetAttribute(k_stencil_hf, cudaFuncAttributeMaxDynamicSharedMemorySize, 110 * 1024);
  return check_launch();
}

template <int OCC>
static void launch_stencil_kernel(int mode, int prec, bool r64, bool planar, dim3 grid, dim3 block, size_t smem,
                                  cudaStream_t s, const StencilArgs& A) {
  if (prec == PGJ_FP32) {
    if (mode == kPlain && planar) k_stencil<float, kPlain, OCC, float, true><<<grid, block, smem, s>>>(A);
    else if (mode == kPlain) k_stencil<float, kPlain, OCC><<<grid, block, smem, s>>>(A);
    else if (planar && r64) k_stencil<float, kPCG, OCC, double, true><<<grid, block, smem, s>>>(A);
    else if (planar) k_stencil<float, kPCG, OCC, float, true><<<grid, block, smem, s>>>(A);
    else if (r64) k_stencil<float, kPCG, OCC, double><<<grid, block, smem, s>>>(A);
    else k_stencil<float, kPCG, OCC><<<grid, block, smem, s>>>(A);
  } else {
    if (mode == kPlain) k_stencil<double, kPlain, OCC><<<grid, block, smem, s>>>(A);
    else if (mode == kPCG) k_stencil<double, kPCG, OCC><<<grid, block, smem, s>>>(A);
    else k_stencil<double, kResidual, OCC><<<grid, block, smem, s>>>(A);
  }
}

int launch_stencil(pgj_ctx* c, int mode, int loads, int prec, const void* in, void* out, const double* f,
                   const int32_t* active_ext, cudaStream_t s, const LoadScalars* rel_flags, bool planar_plain) {
  const int n = c->n;
  StencilArgs A;
  A.n = n; A.ty = c->sg.ty; A.zc = c->sg.zc;
  A.lpd = c->lpd;
  A.a = c->a; A.in = in; A.out = out; A.f = f; A.active_ext = active_ext;
  A.scal = c->scal; A.partials = c->partials; A.kc = c->kc; A.iteration_cap = c->cap;
  A.err = c->cond + 2;
  A.rel_flags = rel_flags;
  const size_t tsz = prec == PGJ_FP32 ? 4 : 8;
  // the FP32 recurrence vectors of a slab-fused context are component-planar, (3, N) per load: the
  // operator writes its q that way (p is read interleaved)
  const bool planar = prec == PGJ_FP32 && c->fused && (mode == kPCG || (mode == kPlain && planar_plain));
  // TMA rows need 16-byte aligned starts and sizes: (3 n * element size) % 16 == 0 and an aligned base
  const size_t rowb = 3 * size_t(n) * tsz;
  A.tma = (rowb % 16 == 0) && (reinterpret_cast<uintptr_t>(in) % 16 == 0) ? 1 : 0;
  dim3 grid(c->sg.ntiles, c->sg.nchunks, loads), block(n, c->sg.ty + 1);
  A.stages = A.tma ? c->sg.stages : 2;
  // FP32 recurrence operator with FP64 arithmetic (high-contrast mixed solves)
  const bool r64 = prec == PGJ_FP32 && mode == kPCG && c->op64;
  const size_t rsz = r64 ? 8 : tsz;  // corner exchange in the arithmetic type
  const size_t smem = tsz * size_t(A.stages) * (c->sg.ty + 2) * 3 * n + rsz * 2 * 9 * (c->sg.ty + 1) * n +
                      32 * 4 * 8 + 16 + 8 * A.stages + 64;
  if (c->sg.ntiles * c->sg.nchunks > kMaxPartials) return PGJ_ERR_UNSUPPORTED;
  if (mode != kPlain && mode != kPCG && !(mode == kResidual && prec == PGJ_FP64)) return PGJ_ERR_ARGUMENT;
  // the occupancy variant applies to the recurrence operator; the residual keeps the wide form
  const bool occ3 = c->sg.occ == 3 && mode != kResidual && n * (c->sg.ty + 1) <= 256 && smem <= 72 * 1024;
  if (occ3) launch_stencil_kernel<3>(mode, prec, r64, planar, grid, block, smem, s, A);
  else launch_stencil_kernel<1>(mode, prec, r64, planar, grid, block, smem, s, A);
  return check_launch();
}

// --------------------------------------------------------------------------- right-hand side
// f(node) = -V sum over the 8 elements e = node - b of B_c(b)^T (a_e C0 eps), B_c the element-centre
// gradient (+-1/(4h) per axis); same arithmetic as hybrid_kernels.cu:50-68.
__global__ void k_rhs(int n, int loads, int lpd, const double* __restrict__ a, const double* __restrict__ macros,
                      double lam, double mu, double* __restrict__ f) {
  const size_t N = size_t(n) * n * n;
  const size_t node = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int load = blockIdx.y;
  if (node >= N || load >= loads) return;
  a += size_t(load / lpd) * N;  // this load's design
  const int x = int(node % n), y = int((node / n) % n), z = int(node / (size_t(n) * n));
  const double* m = macros + 6 * load;
  // C0 eps (Voigt, engineering shear)
  const double tr = m[0] + m[1] + m[2];
  double s0[6];
  s0[0] = lam * tr + 2 * mu * m[0];
  s0[1] = lam * tr + 2 * mu * m[1];
  s0[2] = lam * tr + 2 * mu * m[2];
  s0[3] = mu * m[3]; s0[4] = mu * m[4]; s0[5] = mu * m[5];
  const double h = 1.0 / n, g = 1.0 / (4 * h), vol = h * h * h;
  double fx = 0, fy = 0, fz = 0;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const int ex = wrapi(x - (b & 1), n), eyy = wrapi(y - ((b >> 1) & 1), n), ez = wrapi(z - ((b >> 2) & 1), n);
    const double ae = a[(size_t(ez) * n + eyy) * n + ex];
    const double dx = (b & 1) ? g : -g, dy = (b & 2) ? g : -g, dz = (b & 4) ? g : -g;
    double s[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) s[k] = ae * s0[k];
    fx -= vol * (dx * s[0] + dy * s[5] + dz * s[4]);
    fy -= vol * (dx * s[5] + dy * s[1] + dz * s[3]);
    fz -= vol * (dx * s[4] + dy * s[3] + dz * s[2]);
  }
  double* o = f + size_t(load) * 3 * N + 3 * node;
  o[0] = fx; o[1] = fy; o[2] = fz;
}

int launch_rhs(pgj_ctx* c, int loads, const double* macros_dev, double* f, cudaStream_t s) {
  const size_t N = size_t(c->N);
  dim3 grid(unsigned((N + 255) / 256), loads);
  k_rhs<<<grid, 256, 0, s>>>(c->n, loads, c->lpd, c->a, macros_dev, c->lam, c->mu, f);
  return check_launch();
}

// --------------------------------------------------------------------------- norms / targets
// ||f|| per load, target^2 = max(rtol ||f||, 1e-13/sqrt(n))^2; resets iteration counters and
// latches (resident.py:187-191).
__global__ void k_norms(int n, const double* __restrict__ f, double rtol, LoadScalars* scal, double* partials) {
  const size_t N3 = 3 * size_t(n) * n * n;
  const int load = blockIdx.y;
  const double* fl = f + size_t(load) * N3;
  double acc[1] = {0.0};
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N3; i += size_t(gridDim.x) * blockDim.x) {
    const double v = fl[i];
    acc[0] += v * v;
  }
  __shared__ double red[32];
  block_sum<1>(acc, red);
  double* part = partials + size_t(load) * kPartialQ * kMaxPartials;
  if (threadIdx.x == 0) part[blockIdx.x] = acc[0];
  LoadScalars& S = scal[load];
  if (!last_block(&S.ticket[kTicketAux], gridDim.x)) return;
  if (threadIdx.x < 32) {
    const double s2 = warp_sum_partials(part, gridDim.x);
    if (threadIdx.x == 0) {
      const double norm = sqrt(s2);
      const double t = fmax(norm * rtol, 1e-13 / sqrt(double(n)));
      S.norm = norm;
      S.target2 = t * t;
      S.iterations = 0;
      S.total_iterations = 0;
      S.touched = 0;
      S.bad = 0;
      S.failed = 0;
      S.active = 0;
      S.frozen = 0;
      S.restarts = 0;
    }
  }
}

int launch_norms(pgj_ctx* c, int loads, const double* f, double rtol, cudaStream_t s) {
  dim3 grid(148, loads);
  k_norms<<<grid, 256, 0, s>>>(c->n, f, rtol, c->scal, c->partials);
  return check_launch();
}

// --------------------------------------------------------------------------- projection of u
// mean over nodes per component, then subtract (certification projection, resident.py:133-134).
__global__ void k_mean3(int n, const double* __restrict__ u, int which, LoadScalars* scal, double* partials) {
  const size_t N = size_t(n) * n * n;
  const int load = blockIdx.y;
  if (which == 0 && scal[load].frozen) return;  // certification of a design that took its last attempt
  const double* ul = u + size_t(load) * 3 * N;
  double acc[3] = {0.0, 0.0, 0.0};
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
    acc[0] += ul[3 * i]; acc[1] += ul[3 * i + 1]; acc[2] += ul[3 * i + 2];
  }
  __shared__ double red[96];
  block_sum<3>(acc, red);
  double* part = partials + size_t(load) * kPartialQ * kMaxPartials;
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) part[k * kMaxPartials + blockIdx.x] = acc[k];
  LoadScalars& S = scal[load];
  if (!last_block(&S.ticket[kTicketAux], gridDim.x)) return;
  if (threadIdx.x < 32) {
    double v[3];
    for (int k = 0; k < 3; ++k) v[k] = warp_sum_partials(part + k * kMaxPartials, gridDim.x);
    if (threadIdx.x == 0) {
      double* dst = which ? S.mean_r : S.mean_u;
      for (int k = 0; k < 3; ++k) dst[k] = v[k] / double(N);
    }
  }
}

__global__ void k_sub_mean3(int n, double* __restrict__ u, const LoadScalars* scal) {
  const size_t N3 = 3 * size_t(n) * n * n;
  const int load = blockIdx.y;
  if (scal[load].frozen) return;
  double* ul = u + size_t(load) * N3;
  const double m0 = scal[load].mean_u[0], m1 = scal[load].mean_u[1], m2 = scal[load].mean_u[2];
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N3; i += size_t(gridDim.x) * blockDim.x) {
    const int c = int(i % 3);
    ul[i] -= (c == 0 ? m0 : (c == 1 ? m1 : m2));
  }
}

int launch_mean3(pgj_ctx* c, int loads, const double* v, int which, cudaStream_t s) {
  dim3 grid(148, loads);
  k_mean3<<<grid, 256, 0, s>>>(c->n, v, which, c->scal, c->partials);
  return check_launch();
}

int launch_project_u(pgj_ctx* c, int loads, double* u, cudaStream_t s) {
  int st = launch_mean3(c, loads, u, 0, s);
  if (st) return st;
  dim3 grid2(296, loads);
  k_sub_mean3<<<grid2, 256, 0, s>>>(c->n, u, c->scal);
  return check_launch();
}

// --------------------------------------------------------------------------- diagonal scaling
// log d(node, c), d = sum_b a(node - b) diag(Ke)[b][c]; partial sums of log d for the mean.
__global__ void k_logdiag(int n, const double* __restrict__ a, const double* __restrict__ ed, double* __restrict__ out,
                          LoadScalars* scal, double* partials) {
  const size_t N = size_t(n) * n * n;
  double acc[1] = {0.0};
  for (size_t node = size_t(blockIdx.x) * blockDim.x + threadIdx.x; node < N; node += size_t(gridDim.x) * blockDim.x) {
    const int x = int(node % n), y = int((node / n) % n), z = int(node / (size_t(n) * n));
    double d[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const int ex = wrapi(x - (b & 1), n), eyy = wrapi(y - ((b >> 1) & 1), n), ez = wrapi(z - ((b >> 2) & 1), n);
      const double ae = a[(size_t(ez) * n + eyy) * n + ex];
#pragma unroll
      for (int c = 0; c < 3; ++c) d[c] += ae * ed[3 * b + c];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double q = log(d[c]);
      out[3 * node + c] = q;
      acc[0] += q;
    }
  }
  __shared__ double red[32];
  block_sum<1>(acc, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc[0];
  if (!last_block(&scal[0].ticket[kTicketAux2], gridDim.x)) return;
  if (threadIdx.x < 32) {
    const double s2 = warp_sum_partials(partials, gridDim.x);
    if (threadIdx.x == 0) partials[kMaxPartials - 1] = s2 / double(3 * N);
  }
}

__global__ void k_exp_scale(size_t count, double* __restrict__ q, const double* __restrict__ mean, double coef) {
  const double m = *mean;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += size_t(gridDim.x) * blockDim.x)
    q[i] = exp(coef * (q[i] - m));
}

__global__ void k_fill(size_t count, double* __restrict__ q, double v) {
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += size_t(gridDim.x) * blockDim.x) q[i] = v;
}

// diag(Ke) per local node b (bit order), 2x2x2 Gauss, isotropic C0; host-side constant.
void element_diagonal(int n, double lam, double mu, double* ed) {
  const double g = 1.0 / std::sqrt(3.0);
  for (int i = 0; i < 24; ++i) ed[i] = 0.0;
  for (int q = 0; q < 8; ++q) {
    const double p[3] = {0.5 + ((q & 1) ? 0.5 : -0.5) * g, 0.5 + ((q & 2) ? 0.5 : -0.5) * g,
                         0.5 + ((q & 4) ? 0.5 : -0.5) * g};
    for (int b = 0; b < 8; ++b) {
      const int v[3] = {b & 1, (b >> 1) & 1, (b >> 2) & 1};
      double fac[3], grad[3];
      for (int d = 0; d < 3; ++d) fac[d] = v[d] ? p[d] : 1 - p[d];
      for (int d = 0; d < 3; ++d) {
        double prod = 1.0;
        for (int e = 0; e < 3; ++e) if (e != d) prod *= fac[e];
        grad[d] = (2 * v[d] - 1) * prod * n;
      }
      // diagonal of B^T C B for the x, y, z dofs of node b
      const double l2m = lam + 2 * mu;
      ed[3 * b + 0] += l2m * grad[0] * grad[0] + mu * (grad[1] * grad[1] + grad[2] * grad[2]);
      ed[3 * b + 1] += l2m * grad[1] * grad[1] + mu * (grad[0] * grad[0] + grad[2] * grad[2]);
      ed[3 * b + 2] += l2m * grad[2] * grad[2] + mu * (grad[0] * grad[0] + grad[1] * grad[1]);
    }
  }
  const double vol8 = 1.0 / (double(n) * n * n) / 8.0;
  for (int i = 0; i < 24; ++i) ed[i] *= vol8;
}

// s32[c][node] = float(s[3 node + c])
__global__ void k_scale32(size_t N, const double* __restrict__ s, float* __restrict__ s32) {
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
    const double a = s[3 * i], b = s[3 * i + 1], c = s[3 * i + 2];
    s32[i] = float(a);
    s32[N + i] = float(b);
    s32[2 * N + i] = float(c);
  }
}

int launch_scale32(pgj_ctx* c, cudaStream_t s) {
  k_scale32<<<296, 256, 0, s>>>(size_t(c->N), c->scale, c->scale32);
  return check_launch();
}

int launch_scale(pgj_ctx* c, double alpha, cudaStream_t s) {
  const size_t count = 3 * size_t(c->N);
  if (alpha == 0.0) {
    k_fill<<<296, 256, 0, s>>>(count, c->scale, 1.0);
    return check_launch();
  }
  double* edd = c->aux;  // 24 diagonal entries, staged once in the context's aux block
  if (!c->diag_staged) {
    double ed[24];
    element_diagonal(c->n, c->lam, c->mu, ed);
    cudaError_t e = cudaMemcpyAsync(edd, ed, sizeof(ed), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_cuda_error(e);
    c->diag_staged = 1;
  }
  k_logdiag<<<296, 256, 0, s>>>(c->n, c->a, edd, c->scale, c->scal, c->aux + kAuxPartials);
  int st = check_launch();
  if (st) return st;
  k_exp_scale<<<296, 256, 0, s>>>(count, c->scale, c->aux + kAuxPartials + kMaxPartials - 1, -0.5 * alpha);
  return check_launch();
}

}  // namespace pgj
