// Green apply z = P(s . G(s . P r)) with hand-written shared-memory FFTs.
//
// G is the FI HEX8 Green operator of the homogeneous medium C0 on the periodic grid: a real
// 3D DFT of each displacement component, multiplication by the real symmetric 3x3 Fourier symbol
// (6 coefficients per half-spectrum point, 1/N folded in), and the unnormalised inverse DFT
// (the reference uses cuFFT via torch.fft.rfftn/irfftn: exp/asg_gpu_resident_20261103/resident.py:109-117,
// spectral_three in scalar_fi.cu:38-44). Here the transform is five passes over the half
// spectrum, each a batch of 1D FFTs in shared memory (Stockham autosort, radices 2,3,4,5,8):
//   FX : v = s.(r - mean r) per row, two real rows packed into one complex FFT, R2C split.
//   FY : complex FFT along y.
//   FZ : complex FFT along z, symbol multiply, the Parseval form <v, G v> (= r.z), inverse along z.
//   IFY: inverse along y.
//   IFX: C2R along x (two rows per complex FFT), s.w and its per-component sums (projection P).
// Loads whose recurrence is inactive are skipped block-uniformly.
#include "pgj_fft_engine.cuh"
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>
#include <array>
#include <tuple>
#include <vector>

namespace pgj {

bool make_fft_plan(int n, FFTPlan* plan) {
  plan->n = n;
  plan->nst = 0;
  // powers of two as radix-8 stages, except that 2^(3k+1) takes 8^(k-1) * 4 * 4 rather than 8^k * 2
  // (a radix-2 stage has n/2 butterflies per line and sizes the block for itself while the radix-8
  // stage leaves most threads idle: n = 48 as 8 * 2 * 3 vs 4 * 4 * 3)
  int m = n, e = 0;
  while (m % 2 == 0) { m /= 2; ++e; }
  int n8 = e / 3, n4 = e % 3 == 2 ? 1 : 0, n2 = 0;
  if (e % 3 == 1) {
    if (n8 >= 1) { n8 -= 1; n4 = 2; } else { n2 = 1; }
  }
  for (int i = 0; i < n8 && plan->nst < kMaxStages; ++i) plan->radix[plan->nst++] = 8;
  for (int i = 0; i < n4 && plan->nst < kMaxStages; ++i) plan->radix[plan->nst++] = 4;
  for (int i = 0; i < n2 && plan->nst < kMaxStages; ++i) plan->radix[plan->nst++] = 2;
  while (m % 3 == 0 && plan->nst < kMaxStages) { plan->radix[plan->nst++] = 3; m /= 3; }
  while (m % 5 == 0 && plan->nst < kMaxStages) { plan->radix[plan->nst++] = 5; m /= 5; }
  int ns = 1;
  for (int i = 0; i < plan->nst; ++i) {
    plan->ns_div[i] = make_fastdiv(unsigned(ns));
    plan->nb_div[i] = make_fastdiv(unsigned(n / plan->radix[i]));
    ns *= plan->radix[i];
  }
  return m == 1 && n % 2 == 0 && n >= 4;
}

// smem budget per block for the line buffers (two ping-pong buffers)
static constexpr size_t kFFTSmemBudget = 200 * 1024;

FFTGeom fft_geom(int n, int elem_bytes, const FFTPlan& plan, int rb_req, int nky_req, int nkz_req) {
  FFTGeom g;
  const size_t cb = 2 * size_t(elem_bytes);  // complex bytes
  const size_t line = size_t(n + 1) * cb;
  const int ns = n / 2 + 1;
  // butterflies per line in the widest stage; threads along y of every block
  int minr = 8;
  for (int i = 0; i < plan.nst; ++i) minr = plan.radix[i] < minr ? plan.radix[i] : minr;
  const int nb = n / minr;
  auto by_for = [&](int lines) {
    int by = nb;
    while (by > 1 && lines * by > 512) by = (by + 1) / 2;
    return by;
  };
  // tuning overrides (sweeps): PGJ_FFT_RB rows per x block, PGJ_FFT_NKY / PGJ_FFT_NKZ column chunks
  auto env = [](const char* k, int dflt) {
    const char* v = std::getenv(k);
    return v ? std::atoi(v) : dflt;
  };
  // x passes: rb rows (z,y) -> 3 rb / 2 complex lines, rb | n*n, at most ~48 lines
  int rb = env("PGJ_FFT_RB", rb_req > 0 ? rb_req : 16);
  while (rb > 2 && ((size_t(n) * n) % rb != 0 || 2 * (3 * size_t(rb) / 2) * line > kFFTSmemBudget ||
                    3 * rb / 2 > 512))
    rb /= 2;
  g.rb = rb;
  // y and z passes: tiles of kx columns (lines with pitch n+1 in shared memory)
  const size_t budget_y = 200 * 1024, budget_z = 200 * 1024;
  int nky = env("PGJ_FFT_NKY", nky_req > 0 ? nky_req : 1);
  while (nky < ns && ((ns + nky - 1) / nky > 64 || 2 * size_t((ns + nky - 1) / nky) * line > budget_y)) ++nky;
  g.kcy = (ns + nky - 1) / nky;
  g.nky = (ns + g.kcy - 1) / g.kcy;
  int nkz = env("PGJ_FFT_NKZ", nkz_req > 0 ? nkz_req : 1);
  while (nkz < ns && (3 * ((ns + nkz - 1) / nkz) > 48 || 2 * 3 * size_t((ns + nkz - 1) / nkz) * line > budget_z)) ++nkz;
  g.kcz = (ns + nkz - 1) / nkz;
  g.nkz = (ns + g.kcz - 1) / g.kcz;
  g.by_x = by_for(3 * g.rb / 2);
  g.by_y = by_for(g.kcy);
  g.by_z = by_for(3 * g.kcz);
  g.thr_x = 3 * g.rb / 2 * g.by_x;
  g.thr_y = g.kcy * g.by_y;
  g.thr_z = 3 * g.kcz * g.by_z;
  g.div_3n = make_fastdiv(unsigned(3 * n));
  g.div_ns = make_fastdiv(unsigned(ns));
  g.div_n = make_fastdiv(unsigned(n));
  g.div_kcz = make_fastdiv(unsigned(g.kcz));
  return g;
}

struct GreenArgs {
  int n, ns, nsp;  // grid edge, half-spectrum length, padded (even) spectrum row length
  int lpd;         // loads per design: load l uses the scale field (and DFT(s)) of design l / lpd
  FFTPlan plan;
  FFTGeom geo;
  const void* r;         // (L,3N) T input residual
  const double* scale;   // (designs, 3N) fp64 scale field
  void* spec;            // (L,3,n,n,ns) complex T
  const void* sym;       // (6,Nh) T symbol
  const void* tw;        // n complex T twiddles (forward)
  void* sw;              // (L,3N) T output s.w
  LoadScalars* scal;
  double* partials;
  int skip_inactive;     // skip loads whose scal.active == 0 (recurrence use)
  int use_mean;          // subtract scal.mean_r before scaling (projection P of the input)
  int init;              // FZ finalizer: initialise rz instead of forming beta
  int finalize_fz;       // FZ last block forms rz / beta (recurrence use only)
  // slab-fused recurrence (the x/y transforms run in the PCG update kernels): the spectrum holds
  // DFT(s.r); FZ subtracts mean_r . shat (shat = DFT(s)) and forms mean(s.w) by Parseval
  const void* shat;      // (designs, 3, n, n, nsp) complex T: DFT of each component of the scale field
  int fused;
  int forward_only;      // FZ: forward transform along z only (builds shat)
  int unit_input;        // FX: transform s itself (r ignored; builds shat)
  const float4* axis;    // per-axis symbol factors (m, v, d), FP32 z pass at n = 64
  int flex;              // flexible beta: beta = (rz_new - r_new . z_prev) / rz
  double lam, mu;
};

__device__ __forceinline__ bool load_on(const GreenArgs& A, int load) {
  return A.skip_inactive ? (A.scal[load].active != 0) : true;
}

// ---------------------------------------------------------------------------- FX
// block (3 rb/2 lines, by): rows (z,y) row0..row0+rb of one load; two real rows per complex line.
template <typename T>
__global__ void __launch_bounds__(512) k_fx(const GreenArgs A) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int load = blockIdx.y;
  if (!load_on(A, load)) return;
  const int n = A.n, ns = A.ns, rb = A.geo.rb, pitch = n + 1;
  const int tid = flat_tid(), nthr = block_threads();
  const int nl = 3 * rb / 2;  // complex lines
  C* b0 = reinterpret_cast<C*>(smem_raw);
  C* b1 = b0 + nl * pitch;
  const size_t N = size_t(n) * n * n;
  const size_t row0 = size_t(blockIdx.x) * rb;
  const T* r = reinterpret_cast<const T*>(A.r) + size_t(load) * 3 * N;
  const double* sc = A.scale + size_t(load / A.lpd) * 3 * N;
  T m[3] = {T(0), T(0), T(0)};
  if (A.use_mean) { m[0] = T(A.scal[load].mean_r[0]); m[1] = T(A.scal[load].mean_r[1]); m[2] = T(A.scal[load].mean_r[2]); }
  const int total = rb * 3 * n;
  const size_t gbase = row0 * n * 3;
  batched_copy<4>(tid, nthr, total, [&](int i) {
    const size_t g = gbase + i;
    const int c = i % 3;
    const T mc = c == 0 ? m[0] : (c == 1 ? m[1] : m[2]);
    return A.unit_input ? T(sc[g]) : T(sc[g]) * (r[g] - mc);
  }, [&](int i, T v) {
    const int rl = fdiv(i, A.geo.div_3n);
    const int rem = i - rl * 3 * n;
    const int x = rem / 3, c = rem - 3 * x;
    const int rho = 3 * rl + c;
    T* dst = reinterpret_cast<T*>(b0 + (rho >> 1) * pitch + x);
    dst[rho & 1] = v;
  });
  __syncthreads();
  const C* tw = reinterpret_cast<const C*>(A.tw);
  C* res = fft_line<T>(b0, b1, threadIdx.x * pitch, 1, A.plan, tw, false);
  // split: line rho=2l (real part) and rho=2l+1 (imaginary part)
  const int nsp = A.nsp;
  C* spec = reinterpret_cast<C*>(A.spec) + size_t(load) * 3 * size_t(n) * n * nsp;
  const int tot2 = 3 * rb * ns;
  for (int i = tid; i < tot2; i += nthr) {
    const int rho = fdiv(i, A.geo.div_ns), k = i - rho * ns;
    const int l = rho >> 1;
    const C zk = res[l * pitch + k];
    const C zn = res[l * pitch + (k == 0 ? 0 : n - k)];
    C out;
    if ((rho & 1) == 0) {  // (Z[k] + conj Z[n-k]) / 2
      out.x = T(0.5) * (zk.x + zn.x); out.y = T(0.5) * (zk.y - zn.y);
    } else {               // (Z[k] - conj Z[n-k]) / (2i)
      out.x = T(0.5) * (zk.y + zn.y); out.y = T(0.5) * (zn.x - zk.x);
    }
    const int rl = rho / 3, c = rho - 3 * rl;
    spec[(size_t(c) * n * n + row0 + rl) * nsp + k] = out;
  }
}

// ---------------------------------------------------------------------------- FY / IFY
// block (kcy lines, by): one (load, component, z) plane, kx columns k0..k0+kcy.
template <typename T, bool INV>
__global__ void __launch_bounds__(512) k_fy(const GreenArgs A) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lc = blockIdx.z;  // load * 3 + component
  const int load = lc / 3, c = lc - 3 * load;
  if (!load_on(A, load)) return;
  const int n = A.n, ns = A.ns, nsp = A.nsp, pitch = n + 1, kc = A.geo.kcy;
  const int z = blockIdx.y;
  const int k0 = blockIdx.x * kc;
  const int kn = min(kc, ns - k0);
  const int kl = threadIdx.x;
  C* b0 = reinterpret_cast<C*>(smem_raw);
  C* b1 = b0 + kc * pitch;
  C* plane = reinterpret_cast<C*>(A.spec) + (size_t(load) * 3 + c) * size_t(n) * n * nsp + size_t(z) * n * nsp;
  if (kl < kn)
    batched_copy<8>(threadIdx.y, blockDim.y, n, [&](int y) { return plane[size_t(y) * nsp + k0 + kl]; },
                    [&](int y, C v) { b0[kl * pitch + y] = v; });
  __syncthreads();
  const C* tw = reinterpret_cast<const C*>(A.tw);
  C* res = fft_line<T>(b0, b1, kl < kn ? kl * pitch : -1, 1, A.plan, tw, INV);
  if (kl < kn)
    for (int y = threadIdx.y; y < n; y += blockDim.y) plane[size_t(y) * nsp + k0 + kl] = res[kl * pitch + y];
}

// ---------------------------------------------------------------------------- FZ (+ symbol)
// block (kcz, by, 3): one (load, ky), kx columns k0..k0+kcz, the three components along z.
template <typename T>
__global__ void __launch_bounds__(512) k_fz(const GreenArgs A) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int load = blockIdx.z;
  if (!load_on(A, load)) return;
  const int n = A.n, ns = A.ns, nsp = A.nsp, pitch = n + 1, kc = A.geo.kcz;
  const int ky = blockIdx.y;
  const int k0 = blockIdx.x * kc;
  const int kn = min(kc, ns - k0);
  const int kl = threadIdx.x, c = threadIdx.z;
  const int tid = flat_tid();
  C* b0 = reinterpret_cast<C*>(smem_raw);
  C* b1 = b0 + 3 * kc * pitch;
  double* red = reinterpret_cast<double*>(b1 + 3 * kc * pitch);  // 32 x 4 doubles
  const size_t plane = size_t(n) * n * nsp;  // one component
  C* sp = reinterpret_cast<C*>(A.spec) + size_t(load) * 3 * plane;
  const int line = c * kc + kl;
  if (kl < kn)
    batched_copy<8>(threadIdx.y, blockDim.y, n,
                    [&](int z) { return sp[c * plane + (size_t(z) * n + ky) * nsp + k0 + kl]; },
                    [&](int z, C v) { b0[line * pitch + z] = v; });
  __syncthreads();
  const C* tw = reinterpret_cast<const C*>(A.tw);
  C* res = fft_line<T>(b0, b1, kl < kn ? line * pitch : -1, 1, A.plan, tw, false);
  if (A.forward_only) {
    if (kl < kn)
      for (int z = threadIdx.y; z < n; z += blockDim.y)
        sp[c * plane + (size_t(z) * n + ky) * nsp + k0 + kl] = res[line * pitch + z];
    return;
  }
  // symbol multiply and Parseval partial sums: rows kz over (threadIdx.y, threadIdx.z)
  const T* sym = reinterpret_cast<const T*>(A.sym);
  const C* sh = reinterpret_cast<const C*>(A.shat) + size_t(load / A.lpd) * 3 * plane;
  const size_t Nh = size_t(n) * n * ns;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  if (kl < kn) {
    const int kx = k0 + kl;
    const double wgt = (kx == 0 || kx == n / 2) ? 1.0 : 2.0;
    T m[3] = {T(0), T(0), T(0)};
    if (A.fused) { m[0] = T(A.scal[load].mean_r[0]); m[1] = T(A.scal[load].mean_r[1]); m[2] = T(A.scal[load].mean_r[2]); }
    for (int kz = threadIdx.y + blockDim.y * threadIdx.z; kz < n; kz += blockDim.y * blockDim.z) {
      const size_t kk = (size_t(kz) * n + ky) * ns + kx;
      const T c0 = sym[kk], c1 = sym[Nh + kk], c2 = sym[2 * Nh + kk];
      const T c3 = sym[3 * Nh + kk], c4 = sym[4 * Nh + kk], c5 = sym[5 * Nh + kk];
      C* px = res + (0 * kc + kl) * pitch + kz;
      C* py = res + (1 * kc + kl) * pitch + kz;
      C* pz = res + (2 * kc + kl) * pitch + kz;
      C x = *px, y = *py, zv = *pz;
      C s0, s1, s2;
      if (A.fused) {
        // DFT(s.(r - mean r)) = DFT(s.r) - mean r . DFT(s)
        const size_t ks = (size_t(kz) * n + ky) * nsp + kx;
        s0 = sh[ks]; s1 = sh[plane + ks]; s2 = sh[2 * plane + ks];
        x.x -= m[0] * s0.x; x.y -= m[0] * s0.y;
        y.x -= m[1] * s1.x; y.y -= m[1] * s1.y;
        zv.x -= m[2] * s2.x; zv.y -= m[2] * s2.y;
      }
      C wx, wy, wz;
      wx.x = c0 * x.x + c3 * y.x + c4 * zv.x; wx.y = c0 * x.y + c3 * y.y + c4 * zv.y;
      wy.x = c3 * x.x + c1 * y.x + c5 * zv.x; wy.y = c3 * x.y + c1 * y.y + c5 * zv.y;
      wz.x = c4 * x.x + c5 * y.x + c2 * zv.x; wz.y = c4 * x.y + c5 * y.y + c2 * zv.y;
      acc[0] += wgt * (double(x.x) * wx.x + double(x.y) * wx.y + double(y.x) * wy.x + double(y.y) * wy.y +
                       double(zv.x) * wz.x + double(zv.y) * wz.y);
      if (A.fused) {
        // sum_x s w = sum_k W conj(DFT(s)) (1/N is folded into the symbol)
        acc[1] += wgt * (double(wx.x) * s0.x + double(wx.y) * s0.y);
        acc[2] += wgt * (double(wy.x) * s1.x + double(wy.y) * s1.y);
        acc[3] += wgt * (double(wz.x) * s2.x + double(wz.y) * s2.y);
      }
      *px = wx; *py = wy; *pz = wz;
    }
  }
  __syncthreads();
  C* other = (res == b0) ? b1 : b0;
  C* res2 = fft_line<T>(res, other, kl < kn ? line * pitch : -1, 1, A.plan, tw, true);
  if (kl < kn)
    for (int z = threadIdx.y; z < n; z += blockDim.y)
      sp[c * plane + (size_t(z) * n + ky) * nsp + k0 + kl] = res2[line * pitch + z];
  if (!A.finalize_fz) return;
  const int nblk = gridDim.x * gridDim.y, blk = blockIdx.x + gridDim.x * blockIdx.y;
  double* part = A.partials + size_t(load) * kPartialQ * kMaxPartials;
  if (A.fused) {
    block_sum<4>(acc, red);
    if (tid == 0)
      for (int k = 0; k < 4; ++k) part[k * kMaxPartials + blk] = acc[k];
  } else {
    double a1[1] = {acc[0]};
    block_sum<1>(a1, red);
    if (tid == 0) part[blk] = a1[0];
  }
  LoadScalars& S = A.scal[load];
  if (!last_block(&S.ticket[kTicketFZ], nblk)) return;
  if (tid < 32) {
    const double rzn = warp_sum_partials(part, nblk);
    double mz[3] = {0.0, 0.0, 0.0};
    if (A.fused)
      for (int k = 0; k < 3; ++k) mz[k] = warp_sum_partials(part + (k + 1) * kMaxPartials, nblk);
    if (tid == 0) {
      if (A.init) {
        S.beta = 0.0;
      } else {
        const double rz = S.rz;
        S.beta = (A.flex ? rzn - S.rz_cross : rzn) / (rz != 0.0 ? rz : 1.0);
      }
      S.rz = rzn;
      if (A.fused)
        for (int k = 0; k < 3; ++k) S.mean_z[k] = mz[k] / double(size_t(n) * n * n);
    }
  }
}

// ---------------------------------------------------------------------------- FZ, n = 64
// z pass of the fused recurrence at n = 64 with the line transforms in registers: a 64-point line
// is an 8 x 8 four-step transform. Lane a of the 8 lanes of a line holds points z = a + 8b; it does
// the 8-point DFT over b, multiplies by w64^(a k2), and a transpose through this warp's shared
// memory hands lane t the values with k2 = t for the 8-point DFT over a; lane t then owns
// kz = t + 8 k1. The inverse runs the same steps backwards. A warp owns four kx columns at one ky
// (all three components); warps never wait on each other, so the only block barrier is the final
// reduction. Same results as k_fz in fused mode (rz, beta and mean(s.w) by Parseval).
constexpr int kFz64Line = 72;                 // complex slots per line (8 rows of 9; conflict-free, as kLine64)

// The FI symbol at (kx, ky, kz) from the per-axis factors (m, v, d) of each wavenumber, the same
// algebra as k_symbol: t = h^3 prod m, trace = t sum (d + v^2), inv_i = 1/(mu trace + (lam+mu) t d_i),
// beta = (lam+mu) t / (1 + sum (lam+mu) t v_i^2 inv_i), cf = (diag(inv) - beta w w^T) / N, w_i = inv_i v_i.
// In FP32 it replaces six scattered loads per wavevector by a few arithmetic instructions.
__device__ __forceinline__ void fi_symbol_f32(const float4& ax, const float4& ay, const float4& az, bool origin,
                                              float lam, float mu, float h3, float invN, float (&cf)[6]) {
  float t = h3 * ax.x;
  t *= ay.x;
  t *= az.x;
  const float trace = ((ax.z + ax.y * ax.y) + (ay.z + ay.y * ay.y) + (az.z + az.y * az.y)) * t;
  const float lm = lam + mu, b = lm * t;
  const float inv0 = origin ? 0.f : __frcp_rn(mu * trace + b * ax.z);
  const float inv1 = origin ? 0.f : __frcp_rn(mu * trace + b * ay.z);
  const float inv2 = origin ? 0.f : __frcp_rn(mu * trace + b * az.z);
  const float den = 1.f + b * ax.y * ax.y * inv0 + b * ay.y * ay.y * inv1 + b * az.y * az.y * inv2;
  const float beta = origin ? 0.f : __fdiv_rn(b, den);
  const float w0 = inv0 * ax.y, w1 = inv1 * ay.y, w2 = inv2 * az.y;
  cf[0] = (inv0 - beta * w0 * w0) * invN;
  cf[1] = (inv1 - beta * w1 * w1) * invN;
  cf[2] = (inv2 - beta * w2 * w2) * invN;
  cf[3] = -beta * w0 * w1 * invN;
  cf[4] = -beta * w0 * w2 * invN;
  cf[5] = -beta * w1 * w2 * invN;
}
constexpr int kFz64Comp = 4 * kFz64Line;      // one component of the warp's four lines

template <typename T, int WPB, int MINB>
__global__ void __launch_bounds__(WPB * 32, MINB) k_fz64(const GreenArgs A) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int N = 64;
  const int load = blockIdx.y;
  if (!load_on(A, load)) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int l = lane >> 3, t = lane & 7;
  const int ns = A.ns, nsp = A.nsp;
  const int groups = (ns + 3) >> 2;
  const int w = blockIdx.x * WPB + warp;
  const int ky = w / groups, kx = (w - ky * groups) * 4 + l;
  const bool valid = ky < N && kx < ns;
  C* buf = reinterpret_cast<C*>(smem_raw) + (warp * 3 * 4 + l) * kFz64Line;  // + c * kFz64Comp
  double* red = reinterpret_cast<double*>(reinterpret_cast<C*>(smem_raw) + WPB * 3 * kFz64Comp);
  const size_t plane = size_t(N) * N * nsp;
  C* sp = reinterpret_cast<C*>(A.spec) + size_t(load) * 3 * plane;
  const C* tw = reinterpret_cast<const C*>(A.tw);
  const C zero = cmk<C>(0.0, 0.0);
  const size_t col = size_t(ky) * nsp + kx;  // offset of (z = 0, ky, kx) in one component
  // forward: DFT over b, twiddle, column write (row k2, column t)
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    C v[8];
#pragma unroll
    for (int b = 0; b < 8; ++b) v[b] = valid ? sp[c * plane + size_t(t + 8 * b) * N * nsp + col] : zero;
    Radix<T, 8>::run(v, false);
#pragma unroll
    for (int k2 = 1; k2 < 8; ++k2) v[k2] = cmul(v[k2], __ldg(&tw[t * k2]));
#pragma unroll
    for (int k2 = 0; k2 < 8; ++k2) buf[c * kFz64Comp + k2 * 9 + t] = v[k2];
  }
  __syncwarp();
  // DFT over a of row t; X[kz = t + 8 k1] goes to (row k1, column t)
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    C v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = buf[c * kFz64Comp + t * 9 + j];
    Radix<T, 8>::run(v, false);
    __syncwarp();  // every lane has read its row before the column writes
#pragma unroll
    for (int k1 = 0; k1 < 8; ++k1) buf[c * kFz64Comp + k1 * 9 + t] = v[k1];
  }
  // symbol multiply and the Parseval sums on the lane's own column
  const T* sym = reinterpret_cast<const T*>(A.sym);
  const C* sh = reinterpret_cast<const C*>(A.shat) + size_t(load / A.lpd) * 3 * plane;
  const size_t Nh = size_t(N) * N * ns;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  if (valid) {
    const double wgt = (kx == 0 || kx == N / 2) ? 1.0 : 2.0;
    const T m0 = T(A.scal[load].mean_r[0]), m1 = T(A.scal[load].mean_r[1]), m2 = T(A.scal[load].mean_r[2]);
    float4 axx = make_float4(0.f, 0.f, 0.f, 0.f), axy = axx;
    const float h3 = 1.f / float(N * N * N), invN = h3;
    if constexpr (sizeof(T) == 4) { axx = A.axis[kx]; axy = A.axis[ky]; }
#pragma unroll 2
    for (int k1 = 0; k1 < 8; ++k1) {
      const int kz = t + 8 * k1;
      T c0, c1, c2, c3, c4, c5;
      if constexpr (sizeof(T) == 4) {
        float cf[6];
        fi_symbol_f32(axx, axy, A.axis[kz], kx == 0 && ky == 0 && kz == 0, float(A.lam), float(A.mu), h3, invN, cf);
        c0 = cf[0]; c1 = cf[1]; c2 = cf[2]; c3 = cf[3]; c4 = cf[4]; c5 = cf[5];
      } else {
        const size_t kk = (size_t(kz) * N + ky) * ns + kx;
        c0 = sym[kk]; c1 = sym[Nh + kk]; c2 = sym[2 * Nh + kk];
        c3 = sym[3 * Nh + kk]; c4 = sym[4 * Nh + kk]; c5 = sym[5 * Nh + kk];
      }
      const size_t ks = size_t(kz) * N * nsp + col;
      const C s0 = sh[ks], s1 = sh[plane + ks], s2 = sh[2 * plane + ks];
      C* px = buf + k1 * 9 + t;
      C x = px[0], y = px[kFz64Comp], zv = px[2 * kFz64Comp];
      x.x -= m0 * s0.x; x.y -= m0 * s0.y;
      y.x -= m1 * s1.x; y.y -= m1 * s1.y;
      zv.x -= m2 * s2.x; zv.y -= m2 * s2.y;
      C wx, wy, wz;
      wx.x = c0 * x.x + c3 * y.x + c4 * zv.x; wx.y = c0 * x.y + c3 * y.y + c4 * zv.y;
      wy.x = c3 * x.x + c1 * y.x + c5 * zv.x; wy.y = c3 * x.y + c1 * y.y + c5 * zv.y;
      wz.x = c4 * x.x + c5 * y.x + c2 * zv.x; wz.y = c4 * x.y + c5 * y.y + c2 * zv.y;
      acc[0] += wgt * (double(x.x) * wx.x + double(x.y) * wx.y + double(y.x) * wy.x + double(y.y) * wy.y +
                       double(zv.x) * wz.x + double(zv.y) * wz.y);
      acc[1] += wgt * (double(wx.x) * s0.x + double(wx.y) * s0.y);
      acc[2] += wgt * (double(wy.x) * s1.x + double(wy.y) * s1.y);
      acc[3] += wgt * (double(wz.x) * s2.x + double(wz.y) * s2.y);
      px[0] = wx; px[kFz64Comp] = wy; px[2 * kFz64Comp] = wz;
    }
  }
  // inverse: DFT over k1 of the own column, twiddle, column write (row a, column t); then the
  // DFT over k2 of row t gives z = t + 8 b
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    C v[8];
#pragma unroll
    for (int k1 = 0; k1 < 8; ++k1) v[k1] = buf[c * kFz64Comp + k1 * 9 + t];
    Radix<T, 8>::run(v, true);
#pragma unroll
    for (int a = 1; a < 8; ++a) {
      C wt = __ldg(&tw[t * a]);
      wt.y = -wt.y;
      v[a] = cmul(v[a], wt);
    }
#pragma unroll
    for (int a = 0; a < 8; ++a) buf[c * kFz64Comp + a * 9 + t] = v[a];
  }
  __syncwarp();
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    C v[8];
#pragma unroll
    for (int k2 = 0; k2 < 8; ++k2) v[k2] = buf[c * kFz64Comp + t * 9 + k2];
    Radix<T, 8>::run(v, true);
    if (valid) {
#pragma unroll
      for (int b = 0; b < 8; ++b) sp[c * plane + size_t(t + 8 * b) * N * nsp + col] = v[b];
    }
  }
  // Parseval partials -> last block: rz, beta, mean(s.w) (as k_fz)
  const int tid = threadIdx.x;
  block_sum<4>(acc, red);
  const int nblk = gridDim.x, blk = blockIdx.x;
  double* part = A.partials + size_t(load) * kPartialQ * kMaxPartials;
  if (tid == 0)
    for (int k = 0; k < 4; ++k) part[k * kMaxPartials + blk] = acc[k];
  LoadScalars& S = A.scal[load];
  if (!last_block(&S.ticket[kTicketFZ], nblk)) return;
  if (tid < 32) {
    const double rzn = warp_sum_partials(part, nblk);
    double mz[3];
    for (int k = 0; k < 3; ++k) mz[k] = warp_sum_partials(part + (k + 1) * kMaxPartials, nblk);
    if (tid == 0) {
      if (A.init) {
        S.beta = 0.0;
      } else {
        const double rz = S.rz;
        S.beta = (A.flex ? rzn - S.rz_cross : rzn) / (rz != 0.0 ? rz : 1.0);
      }
      S.rz = rzn;
      for (int k = 0; k < 3; ++k) S.mean_z[k] = mz[k] / double(size_t(N) * N * N);
    }
  }
}

// ---------------------------------------------------------------------------- IFX
// block (3 rb/2 lines, by): C2R of rb rows, two rows per complex line; s.w and its sums.
template <typename T>
__global__ void __launch_bounds__(512) k_ifx(const GreenArgs A) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int load = blockIdx.y;
  if (!load_on(A, load)) return;
  const int n = A.n, ns = A.ns, rb = A.geo.rb, pitch = n + 1;
  const int tid = flat_tid(), nthr = block_threads();
  const int nl = 3 * rb / 2;
  C* b0 = reinterpret_cast<C*>(smem_raw);
  C* b1 = b0 + nl * pitch;
  double* red = reinterpret_cast<double*>(b1 + nl * pitch);
  const size_t N = size_t(n) * n * n;
  const size_t row0 = size_t(blockIdx.x) * rb;
  const int nsp = A.nsp;
  const C* spec = reinterpret_cast<const C*>(A.spec) + size_t(load) * 3 * size_t(n) * n * nsp;
  // Z[k] = A[k] + i B[k] over the full line, A/B Hermitian-extended; DC/Nyquist imaginary parts dropped
  const int total = nl * n;
  batched_copy<4>(tid, nthr, total, [&](int i) {
    const int l = fdiv(i, A.geo.div_n), k = i - l * n;
    C v[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int rho = 2 * l + h;
      const int rl = rho / 3, c = rho - 3 * rl;
      const C* src = spec + (size_t(c) * n * n + row0 + rl) * nsp;
      C val;
      if (k < ns) {
        val = src[k];
        if (k == 0 || k == n / 2) val.y = T(0);
      } else {
        val = cconj(src[n - k]);
      }
      v[h] = val;
    }
    C z;
    z.x = v[0].x - v[1].y;
    z.y = v[0].y + v[1].x;
    return z;
  }, [&](int i, C z) {
    const int l = fdiv(i, A.geo.div_n), k = i - l * n;
    b0[l * pitch + k] = z;
  });
  __syncthreads();
  const C* tw = reinterpret_cast<const C*>(A.tw);
  C* res = fft_line<T>(b0, b1, threadIdx.x * pitch, 1, A.plan, tw, true);
  T* sw = reinterpret_cast<T*>(A.sw) + size_t(load) * 3 * N;
  const double* sc = A.scale + size_t(load / A.lpd) * 3 * N;
  double acc[3] = {0.0, 0.0, 0.0};
  const int tot2 = rb * 3 * n;
  const size_t gbase = row0 * n * 3;
  for (int i = tid; i < tot2; i += nthr) {
    const int rl = fdiv(i, A.geo.div_3n);
    const int rem = i - rl * 3 * n;
    const int x = rem / 3, c = rem - 3 * x;
    const int rho = 3 * rl + c;
    const C zz = res[(rho >> 1) * pitch + x];
    const T w = (rho & 1) ? zz.y : zz.x;
    const T o = T(sc[gbase + i]) * w;
    sw[gbase + i] = o;
    const double od = double(o);
    acc[0] += c == 0 ? od : 0.0;
    acc[1] += c == 1 ? od : 0.0;
    acc[2] += c == 2 ? od : 0.0;
  }
  block_sum<3>(acc, red);
  const int nblk = gridDim.x;
  double* part = A.partials + size_t(load) * kPartialQ * kMaxPartials + kMaxPartials;
  if (tid == 0)
    for (int k = 0; k < 3; ++k) part[k * kMaxPartials + blockIdx.x] = acc[k];
  LoadScalars& S = A.scal[load];
  if (!last_block(&S.ticket[kTicketIFX], nblk)) return;
  if (tid < 32) {
    double v[3];
    for (int k = 0; k < 3; ++k) v[k] = warp_sum_partials(part + k * kMaxPartials, nblk);
    if (tid == 0)
      for (int k = 0; k < 3; ++k) S.mean_z[k] = v[k] / double(N);
  }
}

// ---------------------------------------------------------------------------- host side
static size_t smem_x(const pgj_ctx* c, size_t cb) {
  const int nl = 3 * c->fg.rb / 2;
  return 2 * size_t(nl) * (c->n + 1) * cb + 32 * 3 * 8 + 64;
}
static size_t smem_y(const pgj_ctx* c, size_t cb) { return 2 * size_t(c->fg.kcy) * (c->n + 1) * cb; }
static size_t smem_z(const pgj_ctx* c, size_t cb) { return 2 * 3 * size_t(c->fg.kcz) * (c->n + 1) * cb + 32 * 4 * 8 + 64; }

template <typename T> constexpr int fz64_warps() { return sizeof(T) == 4 ? 8 : 4; }  // warps per block
template <typename T>
static size_t fz64_smem() { return size_t(fz64_warps<T>()) * 3 * kFz64Comp * 2 * sizeof(T) + 32 * 4 * 8 + 64; }

template <typename T>
static int run_fz64(pgj_ctx* c, int loads, const GreenArgs& A, cudaStream_t s) {
  constexpr int WPB = fz64_warps<T>();
  const int warps = ((c->ns + 3) / 4) * c->n;  // per load
  const dim3 grid((warps + WPB - 1) / WPB, loads);
  // blocks per SM the register budget is sized for: default three; PGJ_FZ64_MINB = 1 (unbounded), 4, 6
  const char* e = std::getenv("PGJ_FZ64_MINB");
  const int minb = e ? std::atoi(e) : 3;
  if (minb == 1) k_fz64<T, WPB, 1><<<grid, WPB * 32, fz64_smem<T>(), s>>>(A);
  else if (minb == 4) k_fz64<T, WPB, 4><<<grid, WPB * 32, fz64_smem<T>(), s>>>(A);
  else if (minb == 6) k_fz64<T, WPB, 6><<<grid, WPB * 32, fz64_smem<T>(), s>>>(A);
  else k_fz64<T, WPB, 3><<<grid, WPB * 32, fz64_smem<T>(), s>>>(A);
  return check_launch();
}

template <typename T>
static int set_smem_limits() {
  const int lim = 220 * 1024;  // below the 227 KB opt-in less the static shared memory
  cudaFuncSetAttribute(k_fx<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fy<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fy<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fz<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_ifx<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fz64<T, fz64_warps<T>(), 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fz64<T, fz64_warps<T>(), 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fz64<T, fz64_warps<T>(), 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fz64<T, fz64_warps<T>(), 6>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  return check_launch();
}

int prepare_fft_kernels() {
  int st = set_smem_limits<double>();
  return st ? st : set_smem_limits<float>();
}

template <typename T>
static int run_green_pass(pgj_ctx* c, int loads, GreenArgs& A, cudaStream_t s, int pass) {
  const size_t cb = 2 * sizeof(T);
  const int n = c->n;
  const FFTGeom& g = c->fg;
  switch (pass) {
    case 0: k_fx<T><<<dim3((n * n) / g.rb, loads), dim3(3 * g.rb / 2, g.by_x), smem_x(c, cb), s>>>(A); break;
    case 1: k_fy<T, false><<<dim3(g.nky, n, 3 * loads), dim3(g.kcy, g.by_y), smem_y(c, cb), s>>>(A); break;
    case 2: k_fz<T><<<dim3(g.nkz, n, loads), dim3(g.kcz, g.by_z, 3), smem_z(c, cb), s>>>(A); break;
    case 3: k_fy<T, true><<<dim3(g.nky, n, 3 * loads), dim3(g.kcy, g.by_y), smem_y(c, cb), s>>>(A); break;
    default: k_ifx<T><<<dim3((n * n) / g.rb, loads), dim3(3 * g.rb / 2, g.by_x), smem_x(c, cb), s>>>(A); break;
  }
  return check_launch();
}

template <typename T>
static int run_green(pgj_ctx* c, int loads, GreenArgs& A, cudaStream_t s) {
  for (int pass = 0; pass < 5; ++pass) {
    const int st = run_green_pass<T>(c, loads, A, s, pass);
    if (st) return st;
  }
  return PGJ_OK;
}

static float4* axis_table(pgj_ctx* c) {
  return reinterpret_cast<float4*>(static_cast<char*>(c->tw) + size_t(c->n) * (sizeof(double2) + sizeof(float2)));
}

static GreenArgs green_args(pgj_ctx* c, int prec, const void* r) {
  GreenArgs A;
  std::memset(&A, 0, sizeof(A));
  A.n = c->n; A.ns = c->ns; A.nsp = c->ns + (c->ns & 1); A.plan = c->plan; A.geo = c->fg;
  A.lpd = c->lpd;
  A.r = r; A.scale = c->scale; A.spec = c->spec;
  A.sym = prec == PGJ_FP32 ? static_cast<const void*>(c->symbol32) : static_cast<const void*>(c->symbol);
  A.tw = prec == PGJ_FP32 ? static_cast<const void*>(static_cast<double2*>(c->tw) + c->n) : c->tw;
  A.sw = c->sw; A.scal = c->scal; A.partials = c->partials;
  A.axis = axis_table(c);
  A.lam = c->lam; A.mu = c->mu;
  A.flex = prec == PGJ_FP32 ? c->flex : 0;  // beta of the FP32 recurrence: flexible form when set
  return A;
}

int launch_green_pass(pgj_ctx* c, int loads, int prec, const void* r, bool init, int pass, cudaStream_t s) {
  GreenArgs A = green_args(c, prec, r);
  A.skip_inactive = 1;
  A.use_mean = 1;
  A.init = init ? 1 : 0;
  A.finalize_fz = 1;
  return prec == PGJ_FP32 ? run_green_pass<float>(c, loads, A, s, pass) : run_green_pass<double>(c, loads, A, s, pass);
}

int launch_green(pgj_ctx* c, int loads, int prec, const void* r, bool init, cudaStream_t s) {
  GreenArgs A = green_args(c, prec, r);
  A.skip_inactive = 1;
  A.use_mean = 1;
  A.init = init ? 1 : 0;
  A.finalize_fz = 1;
  return prec == PGJ_FP32 ? run_green<float>(c, loads, A, s) : run_green<double>(c, loads, A, s);
}

// z pass of the slab-fused iteration (DFT(s.r) in the spectrum; mean r subtracted through shat).
int launch_fz_fused(pgj_ctx* c, int loads, int prec, bool init, cudaStream_t s) {
  GreenArgs A = green_args(c, prec, c->r);
  A.skip_inactive = 1;
  A.init = init ? 1 : 0;
  A.finalize_fz = 1;
  A.fused = 1;
  A.shat = c->shat;
  const char* e = std::getenv("PGJ_FZ64");
  if (c->n == 64 && !(e && e[0] == '0'))  // line transforms in registers (PGJ_FZ64=0: generic pass)
    return prec == PGJ_FP32 ? run_fz64<float>(c, loads, A, s) : run_fz64<double>(c, loads, A, s);
  return prec == PGJ_FP32 ? run_green_pass<float>(c, loads, A, s, 2) : run_green_pass<double>(c, loads, A, s, 2);
}

// shat = DFT(s) per component (in the context precision), through the x, y and forward z passes on
// the spectrum of load 0; called whenever the scale field changes.
int build_shat(pgj_ctx* c, cudaStream_t s) {
  GreenArgs A = green_args(c, c->prec, c->r);
  A.skip_inactive = 0;
  A.use_mean = 0;
  A.unit_input = 1;
  A.forward_only = 1;
  for (int pass = 0; pass < 3; ++pass) {
    const int st = c->prec == PGJ_FP32 ? run_green_pass<float>(c, 1, A, s, pass) : run_green_pass<double>(c, 1, A, s, pass);
    if (st) return st;
  }
  const size_t bytes = 2 * size_t(c->prec == PGJ_FP32 ? 4 : 8) * 3 * size_t(c->n) * c->n * (c->ns + (c->ns & 1));
  const cudaError_t e = cudaMemcpyAsync(c->shat, c->spec, bytes, cudaMemcpyDeviceToDevice, s);
  return e == cudaSuccess ? PGJ_OK : set_cuda_error(e);
}

// z = P(s . w) = s.w - mean(s.w), from the sw buffer and the IFX finalizer's means.
__global__ void k_project_out(int n, const double* __restrict__ sw, double* __restrict__ z, const LoadScalars* scal) {
  const size_t N3 = 3 * size_t(n) * n * n;
  const int load = blockIdx.y;
  const double m0 = scal[load].mean_z[0], m1 = scal[load].mean_z[1], m2 = scal[load].mean_z[2];
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N3; i += size_t(gridDim.x) * blockDim.x) {
    const int cc = int(i % 3);
    z[size_t(load) * N3 + i] = sw[size_t(load) * N3 + i] - (cc == 0 ? m0 : (cc == 1 ? m1 : m2));
  }
}

int launch_green_standalone(pgj_ctx* c, int loads, const double* r, double* z, cudaStream_t s) {
  int st = launch_mean3(c, loads, r, 1, s);  // scal.mean_r
  if (st) return st;
  GreenArgs A = green_args(c, PGJ_FP64, r);
  A.skip_inactive = 0;
  A.use_mean = 1;
  A.finalize_fz = 0;
  if ((st = run_green<double>(c, loads, A, s))) return st;
  k_project_out<<<dim3(296, loads), 256, 0, s>>>(c->n, static_cast<const double*>(c->sw), z, c->scal);
  return check_launch();
}

// Green-apply autotuner: times the five passes (the loads of one design, all active) for candidate
// tile shapes (rows per x block, y-chunks, z-chunks) on the context's buffers; cached per (n, loads
// per design, precision), so batched contexts share the choice with single ones.
static std::mutex g_fft_mutex;
static std::map<std::tuple<int, int, int>, std::pair<FFTGeom, std::array<int, 3>>> g_fft_tuned;

int autotune_fft(pgj_ctx* c, cudaStream_t s) {
  const auto key = std::make_tuple(c->n, c->lpd, c->prec);
  {
    std::lock_guard<std::mutex> lock(g_fft_mutex);
    auto it = g_fft_tuned.find(key);
    if (it != g_fft_tuned.end()) {
      c->fg = it->second.first;
      for (int k = 0; k < 3; ++k) c->fft_req[k] = it->second.second[k];
      return PGJ_OK;
    }
  }
  if (std::getenv("PGJ_FFT_RB") || std::getenv("PGJ_FFT_NKY") || std::getenv("PGJ_FFT_NKZ")) return PGJ_OK;
  const int eb = c->prec == PGJ_FP32 ? 4 : 8;
  TileEntry t;
  if (tile_table(c->n, c->prec, &t)) {
    c->fg = fft_geom(c->n, eb, c->plan, t.rb, t.nky, t.nkz);
    c->fft_req[0] = t.rb; c->fft_req[1] = t.nky; c->fft_req[2] = t.nkz;
    std::lock_guard<std::mutex> lock(g_fft_mutex);
    g_fft_tuned[key] = {c->fg, {t.rb, t.nky, t.nkz}};
    return PGJ_OK;
  }
  std::vector<FFTGeom> cands;
  std::vector<std::array<int, 3>> reqs;
  for (int rb : {8, 16})
    for (int nky : {1, 2, 3})
      for (int nkz : {1, 2, 3, 4, 6}) {
        FFTGeom g = fft_geom(c->n, eb, c->plan, rb, nky, nkz);
        bool dup = false;
        for (const FFTGeom& h : cands)
          dup = dup || (h.rb == g.rb && h.kcy == g.kcy && h.kcz == g.kcz);
        if (!dup) { cands.push_back(g); reqs.push_back({rb, nky, nkz}); }
      }
  GreenArgs A = green_args(c, c->prec, c->r);
  A.skip_inactive = 0;
  A.use_mean = 0;
  A.finalize_fz = 0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  FFTGeom best = c->fg;
  std::array<int, 3> best_req = {0, 0, 0};
  float best_ms = 1e30f;
  for (int r = 0; r < 10; ++r)  // bring the clocks up before timing anything
    c->prec == PGJ_FP32 ? run_green<float>(c, c->lpd, A, s) : run_green<double>(c, c->lpd, A, s);
  for (size_t ci = 0; ci < cands.size(); ++ci) {
    const FFTGeom& g = cands[ci];
    c->fg = g;
    A.geo = g;
    int st = c->prec == PGJ_FP32 ? run_green<float>(c, c->lpd, A, s) : run_green<double>(c, c->lpd, A, s);
    if (st) { cudaEventDestroy(e0); cudaEventDestroy(e1); c->fg = best; return st; }
    float ms = 1e30f;
    for (int trial = 0; trial < 2; ++trial) {  // best of two trials of three applies
      cudaEventRecord(e0, s);
      for (int r = 0; r < 3; ++r)
        c->prec == PGJ_FP32 ? run_green<float>(c, c->lpd, A, s) : run_green<double>(c, c->lpd, A, s);
      cudaEventRecord(e1, s);
      cudaEventSynchronize(e1);
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      ms = t < ms ? t : ms;
    }
    if (ms < best_ms) { best_ms = ms; best = g; best_req = reqs[ci]; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->fg = best;
  c->fft_req[0] = best_req[0]; c->fft_req[1] = best_req[1]; c->fft_req[2] = best_req[2];
  std::lock_guard<std::mutex> lock(g_fft_mutex);
  g_fft_tuned[key] = {best, best_req};
  return check_launch();
}

// ---------------------------------------------------------------------------- tables
int init_fft_tables(pgj_ctx* c, cudaStream_t s) {
  const int n = c->n;
  std::vector<double2> t64(n);
  std::vector<float2> t32(n);
  for (int k = 0; k < n; ++k) {
    const long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)n;
    const double cr = (double)cosl(ang), ci = (double)sinl(ang);
    t64[k] = make_double2(cr, ci);
    t32[k] = make_float2((float)cr, (float)ci);
  }
  // per-axis factors of the FI symbol (the same expressions as k_symbol): m = cos^2 + sin^2/3,
  // v = 2 sin cos / (h m), d = 4 sin^4 / (3 h^2 m^2) at the half angle pi k / n
  std::vector<float4> ax(n);
  const double h = 1.0 / n;
  for (int k = 0; k < n; ++k) {
    const double a = 3.14159265358979323846 * k / n, sn = std::sin(a), cs = std::cos(a);
    const double m = cs * cs + sn * sn / 3;
    ax[k] = make_float4(float(m), float(2 * sn * cs / (h * m)), float(4 * (sn * sn) * (sn * sn) / (3 * h * h * m * m)), 0.f);
  }
  cudaError_t e = cudaMemcpyAsync(c->tw, t64.data(), n * sizeof(double2), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(static_cast<double2*>(c->tw) + n, t32.data(), n * sizeof(float2), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(axis_table(c), ax.data(), n * sizeof(float4), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e == cudaSuccess ? PGJ_OK : set_cuda_error(e);
}

// FI HEX8 Green symbol: fi_coeff_kernel (formula_kernels.cu:104-126) with the half-angle tables
// of formula_adapter.py:48-53, expanded densely with 1/N folded in (precision_kernels.cu:57-89).
__global__ void k_symbol(int n, double lam, double mu, double* __restrict__ out, float* __restrict__ out32) {
  const int ns = n / 2 + 1;
  const size_t Nh = size_t(n) * n * ns;
  const size_t k = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= Nh) return;
  const int kx = int(k % ns), ky = int((k / ns) % n), kz = int(k / (size_t(ns) * n));
  const double h = 1.0 / n, pi = 3.14159265358979323846;
  const int kk[3] = {kx, ky, kz};
  double m[3], v[3], d[3];
  double t = h * h * h, trace = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double sn, cs;
    sincos(pi * kk[i] / n, &sn, &cs);
    m[i] = cs * cs + sn * sn / 3;
    t *= m[i];
    v[i] = 2 * sn * cs / (h * m[i]);
    d[i] = 4 * (sn * sn) * (sn * sn) / (3 * h * h * m[i] * m[i]);
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) trace += d[i] + v[i] * v[i];
  trace *= t;
  const double b = (lam + mu) * t;
  double inv[3], den = 1.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    inv[i] = k == 0 ? 0.0 : 1.0 / (mu * trace + (lam + mu) * t * d[i]);
    den += b * v[i] * v[i] * inv[i];
  }
  const double beta = k == 0 ? 0.0 : b / den;
  const double invN = 1.0 / (double(n) * n * n);
  double w[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) w[i] = inv[i] * v[i];
  double cf[6];
  cf[0] = (inv[0] - beta * w[0] * w[0]) * invN;
  cf[1] = (inv[1] - beta * w[1] * w[1]) * invN;
  cf[2] = (inv[2] - beta * w[2] * w[2]) * invN;
  cf[3] = -beta * w[0] * w[1] * invN;
  cf[4] = -beta * w[0] * w[2] * invN;
  cf[5] = -beta * w[1] * w[2] * invN;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    if (out) out[j * Nh + k] = cf[j];
    if (out32) out32[j * Nh + k] = float(cf[j]);
  }
}

int build_symbol(int n, double lam, double mu, double* sym, float* sym32, cudaStream_t s) {
  const size_t Nh = size_t(n) * n * (n / 2 + 1);
  k_symbol<<<unsigned((Nh + 255) / 256), 256, 0, s>>>(n, lam, mu, sym, sym32);
  return check_launch();
}

}  // namespace pgj
