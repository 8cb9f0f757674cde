// Shared-memory Stockham FFT engine (radices 2, 3, 4, 5, 8) used by the Green passes.
//
// Two forms of one stage: `stage` runs the butterflies of the single line a thread owns (threads
// along y split them); `stage_lines` spreads the butterflies of many lines over a flat thread
// range, line index fastest (lines at unit offset, e.g. columns) or butterfly index fastest
// (contiguous rows), so shared-memory accesses of a warp stay on distinct banks.
#pragma once
#include "pgj_internal.h"

namespace pgj {

// ----------------------------------------------------------------------------- radix kernels
// Forward transforms use e^{-2 pi i jk/R}; inverse ones the conjugate (unnormalised).
template <typename C>
__device__ __forceinline__ void dft2(C& a, C& b) { C t = a; a = cadd(t, b); b = csub(t, b); }

template <typename C>
__device__ __forceinline__ void dft4(C& v0, C& v1, C& v2, C& v3, bool inv) {
  C a = cadd(v0, v2), b = csub(v0, v2), c = cadd(v1, v3), d = cmul_mi(csub(v1, v3), inv);
  v0 = cadd(a, c); v2 = csub(a, c); v1 = cadd(b, d); v3 = csub(b, d);
}

template <typename T, int R> struct Radix;

template <typename T> struct Radix<T, 2> {
  using C = cplx<T>;
  static __device__ __forceinline__ void run(C (&v)[2], bool) { dft2(v[0], v[1]); }
};
template <typename T> struct Radix<T, 4> {
  using C = cplx<T>;
  static __device__ __forceinline__ void run(C (&v)[4], bool inv) { dft4(v[0], v[1], v[2], v[3], inv); }
};
template <typename T> struct Radix<T, 8> {
  using C = cplx<T>;
  static __device__ __forceinline__ void run(C (&v)[8], bool inv) {
    const T r2 = T(0.70710678118654752440);
    C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4(e0, e1, e2, e3, inv);
    dft4(o0, o1, o2, o3, inv);
    // twiddles W8^k (forward (1-i)/sqrt2 ...), conjugated for the inverse
    C t1, t2, t3;
    if (!inv) {
      t1.x = r2 * (o1.x + o1.y); t1.y = r2 * (o1.y - o1.x);
      t2.x = o2.y; t2.y = -o2.x;
      t3.x = r2 * (o3.y - o3.x); t3.y = -r2 * (o3.x + o3.y);
    } else {
      t1.x = r2 * (o1.x - o1.y); t1.y = r2 * (o1.x + o1.y);
      t2.x = -o2.y; t2.y = o2.x;
      t3.x = -r2 * (o3.x + o3.y); t3.y = r2 * (o3.x - o3.y);
    }
    v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
    v[1] = cadd(e1, t1); v[5] = csub(e1, t1);
    v[2] = cadd(e2, t2); v[6] = csub(e2, t2);
    v[3] = cadd(e3, t3); v[7] = csub(e3, t3);
  }
};
template <typename T> struct Radix<T, 3> {
  using C = cplx<T>;
  static __device__ __forceinline__ void run(C (&v)[3], bool inv) {
    const T s3 = T(0.86602540378443864676);
    C s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
    C t; t.x = v[0].x - T(0.5) * s.x; t.y = v[0].y - T(0.5) * s.y;
    v[0] = cadd(v[0], s);
    C u = cmul_mi(d, inv); u.x *= s3; u.y *= s3;
    v[1] = cadd(t, u); v[2] = csub(t, u);
  }
};
template <typename T> struct Radix<T, 5> {
  using C = cplx<T>;
  static __device__ __forceinline__ void run(C (&v)[5], bool inv) {
    const T c1 = T(0.30901699437494742410), c2 = T(-0.80901699437494742410);
    const T s1 = T(0.95105651629515357212), s2 = T(0.58778525229247312917);
    C s14 = cadd(v[1], v[4]), d14 = csub(v[1], v[4]), s23 = cadd(v[2], v[3]), d23 = csub(v[2], v[3]);
    C a1, a2, b1, b2;
    a1.x = v[0].x + c1 * s14.x + c2 * s23.x; a1.y = v[0].y + c1 * s14.y + c2 * s23.y;
    a2.x = v[0].x + c2 * s14.x + c1 * s23.x; a2.y = v[0].y + c2 * s14.y + c1 * s23.y;
    b1.x = s1 * d14.x + s2 * d23.x; b1.y = s1 * d14.y + s2 * d23.y;
    b2.x = s2 * d14.x - s1 * d23.x; b2.y = s2 * d14.y - s1 * d23.y;
    v[0] = cadd(v[0], cadd(s14, s23));
    C ib1 = cmul_mi(b1, inv), ib2 = cmul_mi(b2, inv);
    v[1] = cadd(a1, ib1); v[4] = csub(a1, ib1);
    v[2] = cadd(a2, ib2); v[3] = csub(a2, ib2);
  }
};

// One Stockham stage on the line owned by this thread (its elements at stride es from `src` / `dst`),
// butterflies j along threadIdx.y: out[(j/Ns)Ns R + j%Ns + r Ns] = DFT_R over r of
// in[j + r n/R] * W^{r (j%Ns)}, W = e^{-2 pi i/(Ns R)}.
template <typename T, int R>
__device__ __forceinline__ void stage(const cplx<T>* __restrict__ src, cplx<T>* __restrict__ dst, int es, int n,
                                      int Ns, const FastDiv& nsd, const cplx<T>* __restrict__ tw, bool inv) {
  using C = cplx<T>;
  const int nb = n / R;
  const int step = n / (Ns * R);
  for (int j = threadIdx.y; j < nb; j += blockDim.y) {
    const int jq = fdiv(j, nsd);
    const int jm = j - jq * Ns;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[(j + r * nb) * es];
    if (jm) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        C w = tw[r * jm * step];
        if (inv) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    Radix<T, R>::run(v, inv);
    const int base = jq * Ns * R + jm;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[(base + r * Ns) * es] = v[r];
  }
}

// All stages on the thread's line at offset `off` (elements at stride es) of the ping-pong buffers
// b0/b1; off < 0 marks an idle thread (it still joins the barriers). Returns the result buffer.
template <typename T>
__device__ cplx<T>* fft_line(cplx<T>* b0, cplx<T>* b1, int off, int es, const FFTPlan& pl, const cplx<T>* tw,
                             bool inv) {
  cplx<T>* src = b0;
  cplx<T>* dst = b1;
  int Ns = 1;
  for (int st = 0; st < pl.nst; ++st) {
    const int R = pl.radix[st];
    const FastDiv& nsd = pl.ns_div[st];
    if (off >= 0) {
      switch (R) {
        case 8: stage<T, 8>(src + off, dst + off, es, pl.n, Ns, nsd, tw, inv); break;
        case 4: stage<T, 4>(src + off, dst + off, es, pl.n, Ns, nsd, tw, inv); break;
        case 2: stage<T, 2>(src + off, dst + off, es, pl.n, Ns, nsd, tw, inv); break;
        case 3: stage<T, 3>(src + off, dst + off, es, pl.n, Ns, nsd, tw, inv); break;
        default: stage<T, 5>(src + off, dst + off, es, pl.n, Ns, nsd, tw, inv); break;
      }
    }
    __syncthreads();
    cplx<T>* t = src; src = dst; dst = t;
    Ns *= R;
  }
  return src;
}


// Stage over `nl` lines at offsets l * lp (elements at stride es), work items w = tid, tid+nthr, ...
// LFAST: w -> (l = w % nl, j = w / nl); otherwise (l = w / nb, j = w % nb).
template <typename T, int R, bool LFAST>
__device__ __forceinline__ void stage_lines(const cplx<T>* __restrict__ src, cplx<T>* __restrict__ dst, int nl, int lp,
                                            int es, int n, int Ns, const FastDiv& nsd, const FastDiv& div,
                                            const cplx<T>* __restrict__ tw, bool inv, int tid, int nthr) {
  using C = cplx<T>;
  const int nb = n / R;
  const int step = n / (Ns * R);
  const int total = nl * nb;
  for (int w = tid; w < total; w += nthr) {
    int l, j;
    if (LFAST) { j = fdiv(w, div); l = w - j * nl; }
    else { l = fdiv(w, div); j = w - l * nb; }
    const int jq = fdiv(j, nsd);
    const int jm = j - jq * Ns;
    const C* s = src + l * lp;
    C* d = dst + l * lp;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = s[(j + r * nb) * es];
    if (jm) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        C w2 = __ldg(&tw[r * jm * step]);
        if (inv) w2.y = -w2.y;
        v[r] = cmul(v[r], w2);
      }
    }
    Radix<T, R>::run(v, inv);
    const int base = jq * Ns * R + jm;
#pragma unroll
    for (int r = 0; r < R; ++r) d[(base + r * Ns) * es] = v[r];
  }
}

// All stages over `nl` lines, ping-pong between b0 and b1 with one block barrier per stage; returns
// the buffer holding the result. `ldiv` divides by nl (LFAST only).
// Always inlined into the slab kernels, its only callers: as a called function it kept their
// registers and the plan in local memory across the call (a 440-byte stack frame) and made their
// speed depend on how many kernels called it (slab update n = 32: 16.5 vs 24.5 us). The per-line
// fft_line of the unfused passes stays a compiler choice (forced inline it made the z pass slower).
template <typename T, bool LFAST>
__device__ __forceinline__ cplx<T>* fft_lines(cplx<T>* b0, cplx<T>* b1, int nl, int lp, int es, const FFTPlan& pl,
                              const FastDiv& ldiv, const cplx<T>* tw, bool inv, int tid, int nthr) {
  cplx<T>* src = b0;
  cplx<T>* dst = b1;
  int Ns = 1;
  for (int st = 0; st < pl.nst; ++st) {
    const int R = pl.radix[st];
    const FastDiv& nsd = pl.ns_div[st];
    const FastDiv& div = LFAST ? ldiv : pl.nb_div[st];
    switch (R) {
      case 8: stage_lines<T, 8, LFAST>(src, dst, nl, lp, es, pl.n, Ns, nsd, div, tw, inv, tid, nthr); break;
      case 4: stage_lines<T, 4, LFAST>(src, dst, nl, lp, es, pl.n, Ns, nsd, div, tw, inv, tid, nthr); break;
      case 2: stage_lines<T, 2, LFAST>(src, dst, nl, lp, es, pl.n, Ns, nsd, div, tw, inv, tid, nthr); break;
      case 3: stage_lines<T, 3, LFAST>(src, dst, nl, lp, es, pl.n, Ns, nsd, div, tw, inv, tid, nthr); break;
      default: stage_lines<T, 5, LFAST>(src, dst, nl, lp, es, pl.n, Ns, nsd, div, tw, inv, tid, nthr); break;
    }
    __syncthreads();
    cplx<T>* t = src; src = dst; dst = t;
    Ns *= R;
  }
  return src;
}

}  // namespace pgj
