// Internal host-side interfaces shared by the libpgj translation units.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include "pgj_common.cuh"

namespace pgj {

struct FFTPlan {
  int n;
  int nst;
  int radix[kMaxStages];
  FastDiv ns_div[kMaxStages];  // stride Ns of each stage (product of the earlier radices)
  FastDiv nb_div[kMaxStages];  // butterflies per line of each stage (n / radix)
};
bool make_fft_plan(int n, FFTPlan* plan);

// Launch geometry of the streaming stencil for a grid edge n.
struct StencilGeom {
  int ty;      // output node rows per block (block is n x (ty+1) threads)
  int ntiles;  // tiles along y
  int zc;      // output node planes per block
  int nchunks; // chunks along z
  int stages;  // node-plane buffers of the TMA staging pipeline (2..4)
  int occ;     // 1: up to 512 threads per block; 3: at most 256 threads, three blocks per SM
};
StencilGeom stencil_geom(int n, int loads);
StencilGeom stencil_geom_shape(int n, int ty, int zc, int stages = 2, int occ = 1);

// Geometry of the FFT passes.
struct FFTGeom {
  int rb;        // rows (z,y) per x-pass block
  int kcy;       // kx columns per y-pass block
  int nky;       // y-pass chunks
  int kcz;       // kx columns per z-pass block
  int nkz;       // z-pass chunks
  int thr_x, thr_y, thr_z;  // threads per block of the x, y and z passes
  int by_x, by_y, by_z;     // threads along y (butterflies of a line) per pass; x (and z) index lines
  FastDiv div_3n, div_ns, div_n, div_kcz;
};
FFTGeom fft_geom(int n, int elem_bytes, const FFTPlan& plan, int rb_req = 0, int nky_req = 0, int nkz_req = 0);

enum StencilMode { kPlain = 0, kPCG = 1, kResidual = 2 };

struct StencilArgs {
  int n, ty, zc;
  int lpd;                     // loads per design: load l reads the density of design l / lpd
  const double* a;             // (designs, N)
  const void* in;
  void* out;
  const double* f;             // residual mode: right-hand side
  const int32_t* active_ext;   // plain mode: optional external mask
  const LoadScalars* rel_flags; // residual mode: when set, only loads with rel_flags[l].reliable
  LoadScalars* scal;           // pcg / residual modes
  double* partials;            // [load][4][nblk]
  OpConst kc;
  int iteration_cap;
  int tma;                     // stage planes with bulk async copies (aligned rows) instead of cp.async
  int stages;                  // plane buffers in the staging pipeline
  int* err;                    // set to 1 if a bounded device wait expired
  void* qb;                    // halo-free recurrence operator: boundary rows (L, n, ntiles, 3, n)
};

// Partial-sum slots per load per kernel (blocks per load upper bound).
constexpr int kMaxPartials = 4096;
constexpr int kPartialQ = 5;
// aux block: [0,24) stiffness diagonal per local node, [32,68) unit Voigt macros,
// [128, 128 + kMaxPartials) scalar-reduction partials of the scale build.
constexpr int kAuxVoigt = 32;
constexpr int kAuxPartials = 128;
constexpr int kAuxDoubles = kAuxPartials + kMaxPartials;

struct Layout {
  size_t a, scale, scale32, symbol, symbol32, tw, solutions, f, x, r, p, q, sw, spec, shat, partials, scal, macros,
      cond, r64, d, aux, qb, total;
};

struct Graphs;

}  // namespace pgj

struct pgj_ctx {
  int n, L, prec;
  int D, lpd;          // designs and loads per design (L = D * lpd); a plain context has D = 1
  double lam, mu;
  long long N;
  int ns;
  long long Nh;
  pgj::OpConst kc;
  pgj::FFTPlan plan;
  pgj::StencilGeom sg;
  pgj::FFTGeom fg;
  pgj::Layout lay;
  char* base;
  size_t bytes;
  // workspace views (per-design fields are D consecutive blocks)
  double* a;           // (D, N)
  double* scale;       // (D, 3N)
  float* scale32;      // FP32 contexts: (D, 3, N) component-planar FP32 copy of scale (first direction)
  double* symbol;
  float* symbol32;
  void* tw;            // n complex twiddles: double2[n] then float2[n]
  double* solutions;   // (L, 3N) fp64 warm starts
  double* f;           // (L, 3N) fp64 right-hand sides
  double* x;           // (L, 3N) fp64 iterate (plain) / refined solution (mixed)
  void* r;             // (L, 3N) T
  void* p;             // (L, 3N) T
  void* q;             // (L, 3N) T
  void* qb;            // FP32 contexts at n = 64: (L, n, n / hg.ty, 3, n) boundary rows of the halo-free operator
  pgj::StencilGeom hg; // halo-free recurrence operator geometry (FP32 slab-fused contexts)
  int hf;              // FP32 slab-fused recurrences use the halo-free operator (PGJ_HF=0: the halo form)
  void* sw;            // (L, 3N) T  s . w (unprojected preconditioned residual)
  void* spec;          // (L, 3, n, n, nsp) complex T
  void* shat;          // (D, 3, n, n, nsp) complex T: DFT of each component of the scale field
  int fused;           // PCG iteration as operator + slab-fused update/transform kernels
  double* partials;    // (L, kPartialQ * kMaxPartials)
  pgj::LoadScalars* scal;  // L records used by the kernels being launched (outer or inner)
  pgj::LoadScalars* scal_out;  // certification / FP64 recurrence records
  pgj::LoadScalars* scal_in;   // mixed refinement: inner FP32 recurrence records
  void* d;             // mixed: (L, 3N) T inner correction
  double* macros;      // (L, 6) device copy
  int* cond;           // device flags (any active)
  double* r64;         // mixed: fp64 residual (L, 3N)
  double* aux;         // (64 + kMaxPartials) doubles: small staged tables and scalar reductions
  double alpha;
  double inner_rtol;
  double rel_delta2;   // mixed reliable updates: replace r when ||r||^2 < rel_delta2 * anchor (0 = off)
  int mixed_mode;      // 0 reliable-update CG, 1 restarted refinement sweeps
  int op64;            // FP32 contexts: the recurrence operator computes in FP64 (FP32 vectors)
  int cap;             // per-load PCG iteration cap (4000, the reference's, unless set)
  int flex;            // FP32 slab-fused recurrences: flexible (Polak-Ribiere) beta
  int tile_source;     // 0 tuned by timing at creation, 1 tile table, 2 environment override
  int fft_req[3];      // requested FFT tiles (rows per x block, y chunks, z chunks)
  int last_refinements;
  int pending_loads;       // loads of the solve enqueued by pgj_solve_async
  int diag_staged;         // stiffness-diagonal constants copied to aux
  int staged_loads;        // macros already on the device
  double staged_macros[6 * pgj::kMaxTotalLoads];
  double alphas[pgj::kMaxDesigns];  // alpha of each design's scale field
  long long last_launches;
  pgj::Graphs* graphs;
};

namespace pgj {
// operator (pgj_operator.cu)
// planar_plain: plain mode writing q component-planar, as the recurrence operator of a slab-fused FP32
// context does (the tuner)
int launch_stencil(pgj_ctx* c, int mode, int loads, int prec, const void* in, void* out, const double* f,
                   const int32_t* active_ext, cudaStream_t s, const LoadScalars* rel_flags = nullptr,
                   bool planar_plain = false);
// offline-tuned tile shapes per (n, precision)
struct TileEntry { int n, prec, ty, zc, stages, occ, rb, nky, nkz; };
bool tile_table(int n, int prec, TileEntry* out);
int launch_rhs(pgj_ctx* c, int loads, const double* macros_dev, double* f, cudaStream_t s);
int launch_scale(pgj_ctx* c, double alpha, cudaStream_t s);
int launch_project_u(pgj_ctx* c, int loads, double* u, cudaStream_t s);
// per-load component means of a DOF vector into scal.mean_u (which=0) or scal.mean_r (which=1)
int launch_mean3(pgj_ctx* c, int loads, const double* v, int which, cudaStream_t s);
int launch_norms(pgj_ctx* c, int loads, const double* f, double rtol, cudaStream_t s);
// fft / green (pgj_fft.cu)
int init_fft_tables(pgj_ctx* c, cudaStream_t s);
int build_symbol(int n, double lam, double mu, double* sym, float* sym32, cudaStream_t s);
int launch_green(pgj_ctx* c, int loads, int prec, const void* r, bool init, cudaStream_t s);
// one Green pass: 0 fft_x, 1 fft_y, 2 fft_z+symbol, 3 ifft_y, 4 ifft_x
int launch_green_pass(pgj_ctx* c, int loads, int prec, const void* r, bool init, int pass, cudaStream_t s);
int launch_green_standalone(pgj_ctx* c, int loads, const double* r, double* z, cudaStream_t s);
int launch_fz_fused(pgj_ctx* c, int loads, int prec, bool init, cudaStream_t s);
int build_shat(pgj_ctx* c, cudaStream_t s);
// FP32 contexts: scale32 = float(scale), component-planar (pgj_operator.cu)
int launch_scale32(pgj_ctx* c, cudaStream_t s);
// slab-fused iteration (pgj_slab.cu)
enum SlabLaunch { kSlabUpdateL = 0, kSlabInitL = 1, kSlabSyncL = 2 };
bool slab_fits(const pgj_ctx* c);
bool slab_fits_shape(int n, int prec);
// halo-free FP32 recurrence operator (pgj_operator.cu): geometry, launch, and whether a context's
// recurrence uses it (FP32, slab-fused, FP32 arithmetic, not switched off)
StencilGeom hf_geom(int n, int lpd);
int launch_stencil_hf(pgj_ctx* c, int loads, cudaStream_t s);
bool slab_register_path(const pgj_ctx* c, int prec);  // the n = 64 register-transform slab kernels
inline bool uses_hf(const pgj_ctx* c, int prec) {
  return prec == PGJ_FP32 && c->fused && c->hf && !c->op64 && slab_register_path(c, prec);
}
// the recurrence operator q = K p (and alpha = r.z / p.q) of one PCG iteration
int launch_recurrence_operator(pgj_ctx* c, int loads, int prec, cudaStream_t s);
int prepare_slab_kernels();
int launch_fxy(pgj_ctx* c, int loads, int prec, int mode, void* u, cudaStream_t s);
int launch_ifxy(pgj_ctx* c, int loads, int prec, bool init, cudaStream_t s, cudaGraphConditionalHandle h,
                bool set_cond);
// pcg (pgj_pcg.cu)
int launch_update_ur(pgj_ctx* c, int loads, int prec, double* u64, void* uT, cudaStream_t s);
int launch_update_p(pgj_ctx* c, int loads, int prec, bool init, cudaStream_t s, cudaGraphConditionalHandle h,
                    bool set_cond);
int launch_init_mask(pgj_ctx* c, int loads, cudaStream_t s);
// mixed refinement (pgj_pcg.cu): inner residual r = T(r64), d = 0, inner targets and masks;
// then x += d for the loads solved in this sweep
int launch_inner_start(pgj_ctx* c, int loads, double inner_rtol, cudaStream_t s);
int launch_inner_finish(pgj_ctx* c, int loads, cudaStream_t s);
// reliable-update mixed solve (pgj_pcg.cu)
int launch_rel_start(pgj_ctx* c, int loads, cudaStream_t s);
int launch_decide(pgj_ctx* c, int loads, cudaGraphConditionalHandle h, cudaStream_t s);
int launch_rel_cond(pgj_ctx* c, int loads, cudaGraphConditionalHandle h, cudaStream_t s);
int launch_rel_fold(pgj_ctx* c, int loads, bool all, cudaStream_t s);
int launch_rel_sync(pgj_ctx* c, int loads, cudaStream_t s);
// energy (pgj_energy.cu)
int launch_energies(pgj_ctx* c, int loads, const double* u, const double* macros_dev, double* e, cudaStream_t s);
int launch_effective_tensor(pgj_ctx* c, const double* a, const double* u, double* C, double* e, cudaStream_t s);

// Points the context's per-design views (a, scale, scale32, shat) at design d for the lifetime of
// the scope, so that the single-design launchers (scale build, FP32 scale copy, DFT(s)) run on it.
struct DesignScope {
  pgj_ctx* c;
  double* a;
  double* scale;
  float* scale32;
  void* shat;
  DesignScope(pgj_ctx* ctx, int d);
  ~DesignScope();
};

int set_cuda_error(cudaError_t e);
// one-time kernel attributes (dynamic shared memory limits); called at context creation
int prepare_stencil_kernels();
int launch_wait_selftest(int tries, int* flag, cudaStream_t s);
// times candidate tile shapes of the operator on the context's buffers and keeps the fastest
int autotune_stencil(pgj_ctx* c, cudaStream_t s);
// times candidate tile shapes of the Green passes and keeps the fastest
int autotune_fft(pgj_ctx* c, cudaStream_t s);
int prepare_fft_kernels();
inline int check_launch() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PGJ_OK : set_cuda_error(e);
}
}  // namespace pgj
