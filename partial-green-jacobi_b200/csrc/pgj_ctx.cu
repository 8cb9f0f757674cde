// libpgj context, workspace layout, certified solve and the C ABI entry points.
//
// The certified solve follows Resident._solve_batch (exp/asg_gpu_resident_20261103/resident.py:186-209):
// rhs and targets; certify (u <- P u, r = f - K u, ||r||); then up to three attempts of
// [initialise masks and directions; iterate while any load is active; certify], restarting only
// when a certificate fails and no latch forbids it. Each attempt is one CUDA graph: the iteration
// loop is a device-side WHILE conditional node whose condition the last kernel of every iteration
// sets from the per-load masks, so the host only synchronises once per attempt to read the
// certificate (the reference polls active.any() every 4 iterations).
#include "pgj_internal.h"
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

namespace pgj {

static thread_local int g_last_cuda_error = 0;
int set_cuda_error(cudaError_t e) {
  g_last_cuda_error = int(e);
  return PGJ_ERR_LAUNCH;
}

struct Graphs {
  cudaStream_t cap = nullptr;  // private capture stream
  int loads = 0;          // solve graph
  int attempt_loads = 0;  // certification / attempt graphs
  int attempt_mode = -1;
  double inner_rtol = 0.0;
  cudaGraphExec_t cert = nullptr;
  cudaGraphExec_t attempt = nullptr;  // FP64: init + PCG loop + certify; mixed: one refinement sweep
  cudaGraphExec_t solve = nullptr;    // whole certified solve with device-side restarts
  double rtol = 0.0;
  int mode = -1;
  ~Graphs() {
    if (cert) cudaGraphExecDestroy(cert);
    if (attempt) cudaGraphExecDestroy(attempt);
    if (solve) cudaGraphExecDestroy(solve);
    if (cap) cudaStreamDestroy(cap);
  }
};

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

DesignScope::DesignScope(pgj_ctx* ctx, int d) : c(ctx), a(ctx->a), scale(ctx->scale), scale32(ctx->scale32), shat(ctx->shat) {
  const size_t N = size_t(c->N), nsp = size_t(c->ns + (c->ns & 1));
  const size_t tsz = c->prec == PGJ_FP32 ? 4 : 8;
  c->a = a + d * N;
  c->scale = scale + d * 3 * N;
  if (scale32) c->scale32 = scale32 + d * 3 * N;
  c->shat = static_cast<char*>(shat) + d * 2 * tsz * 3 * size_t(c->n) * c->n * nsp;
}

DesignScope::~DesignScope() {
  c->a = a;
  c->scale = scale;
  c->scale32 = scale32;
  c->shat = shat;
}

// D designs of `lpd` loads each: per-design fields (a, scale, scale32, shat) are D blocks, per-load
// fields L = D lpd blocks.
static Layout make_layout(int n, int D, int lpd, int prec) {
  const int L = D * lpd;
  Layout y;
  const size_t N = size_t(n) * n * n, N3 = 3 * N;
  const size_t ns = size_t(n / 2 + 1), Nh = size_t(n) * n * ns;
  const size_t nsp = ns + (ns & 1);  // spectrum rows padded to an even length (16-byte aligned rows)
  const size_t tsz = prec == PGJ_FP32 ? 4 : 8;
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t at = o; o = align_up(o + bytes, 256); return at; };
  y.scal = take(sizeof(LoadScalars) * size_t(2 * L));
  y.macros = take(sizeof(double) * 6 * size_t(L));
  y.cond = take(64);
  y.aux = take(sizeof(double) * kAuxDoubles);
  // twiddles (double2[n], float2[n]) and the per-axis Green factors (float4[n]: m, v, d)
  y.tw = take(size_t(n) * (sizeof(double2) + sizeof(float2) + sizeof(float4)));
  const size_t pslots = size_t(kPartialQ * L > 24 ? kPartialQ * L : 24);
  y.partials = take(sizeof(double) * pslots * kMaxPartials);
  y.a = take(sizeof(double) * N * D);
  y.scale = take(sizeof(double) * N3 * D);
  y.symbol = take(sizeof(double) * 6 * Nh);
  y.symbol32 = take(prec == PGJ_FP32 ? sizeof(float) * 6 * Nh : 0);
  y.solutions = take(sizeof(double) * N3 * L);
  y.f = take(sizeof(double) * N3 * L);
  y.x = take(sizeof(double) * N3 * L);
  y.r64 = take(prec == PGJ_FP32 ? sizeof(double) * N3 * L : 0);
  y.d = take(prec == PGJ_FP32 ? tsz * N3 * L : 0);
  y.r = take(tsz * N3 * L);
  y.p = take(tsz * N3 * L);
  y.q = take(tsz * N3 * L);
  y.sw = take(tsz * N3 * L);
  y.spec = take(2 * tsz * 3 * size_t(n) * n * nsp * L);
  y.shat = take(2 * tsz * 3 * size_t(n) * n * nsp * D);
  y.scale32 = take(prec == PGJ_FP32 ? sizeof(float) * N3 * D : 0);
  // boundary rows of the halo-free FP32 operator: n planes x n / ty tiles x 3n per load, ty >= 2
  y.qb = take(prec == PGJ_FP32 && n == 64 ? sizeof(float) * (N3 / 2 + 3 * size_t(n)) * L : 0);
  y.total = o;
  return y;
}

// ------------------------------------------------------------------------------------ graphs
// certification: u <- P u, r = f - K u (FP64), ||r||, mean r (resident.py:133-136)
static int capture_cert(pgj_ctx* c, int L, cudaStream_t s) {
  int st = launch_project_u(c, L, c->x, s);
  if (st) return st;
  double* r = c->prec == PGJ_FP32 ? c->r64 : static_cast<double*>(c->r);
  LoadScalars* saved = c->scal;
  c->scal = c->scal_out;
  st = launch_stencil(c, kResidual, L, PGJ_FP64, c->x, r, c->f, nullptr, s);
  c->scal = saved;
  return st;
}

// one PCG iteration in the inner precision (resident.py:125-131)
static int capture_iteration(pgj_ctx* c, int L, cudaStream_t s, cudaGraphConditionalHandle h, bool last) {
  const int prec = c->prec;
  int st;
  if ((st = launch_recurrence_operator(c, L, prec, s))) return st;
  if (c->fused) {
    // u += alpha p, r -= alpha q and the x/y transforms of s.r; z pass; inverse x/y and p update
    if ((st = launch_fxy(c, L, prec, kSlabUpdateL, prec == PGJ_FP32 ? c->d : static_cast<void*>(c->x), s))) return st;
    if ((st = launch_fz_fused(c, L, prec, false, s))) return st;
    return launch_ifxy(c, L, prec, false, s, h, last);
  }
  if (prec == PGJ_FP32) st = launch_update_ur(c, L, prec, nullptr, c->d, s);
  else st = launch_update_ur(c, L, prec, c->x, nullptr, s);
  if (st) return st;
  if ((st = launch_green(c, L, prec, c->r, false, s))) return st;
  return launch_update_p(c, L, prec, false, s, h, last);
}

// First direction p = M r of a recurrence (the masks are set): unfused Green + p = z, or the fused
// form, which first refreshes DFT(s) in case the scale field was rewritten through its view.
static long long first_direction_launches(const pgj_ctx* c) {
  // per design DFT(s) (3) [+ FP32 scale], then 3; or Green (5) + p
  return c->fused ? (long long)c->D * (c->prec == PGJ_FP32 ? 4 : 3) + 3 : 6;
}

static int capture_first_direction(pgj_ctx* c, int L, cudaStream_t s) {
  int st;
  if (c->fused) {
    for (int d = 0; d < c->D; ++d) {
      DesignScope view(c, d);
      if ((st = build_shat(c, s))) return st;
      if (c->prec == PGJ_FP32 && (st = launch_scale32(c, s))) return st;
    }
    if ((st = launch_fxy(c, L, c->prec, kSlabInitL, nullptr, s))) return st;
    if ((st = launch_fz_fused(c, L, c->prec, true, s))) return st;
    return launch_ifxy(c, L, c->prec, true, s, 0, false);
  }
  st = launch_green(c, L, c->prec, c->r, true, s);
  return st ? st : launch_update_p(c, L, c->prec, true, s, 0, false);
}

// Appends a conditional node of `type` after the current capture point of `s` and returns its body
// graph; the capture of `s` continues after the node.
static int add_conditional(cudaStream_t s, cudaGraphConditionalHandle* h, unsigned def, cudaGraphConditionalNodeType type,
                           cudaGraph_t* body) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t cg = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  cudaError_t e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &ndeps);
  if (e == cudaSuccess && !*h) e = cudaGraphConditionalHandleCreate(h, cg, def, cudaGraphCondAssignDefault);
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
  cp.conditional.handle = *h;
  cp.conditional.type = type;
  cp.conditional.size = 1;
  cudaGraphNode_t node = nullptr;
  if (e == cudaSuccess) e = cudaGraphAddNode(&node, cg, deps, ndeps, &cp);
  if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies);
  if (e != cudaSuccess) return set_cuda_error(e);
  *body = cp.conditional.phGraph_out[0];
  return PGJ_OK;
}

// Creates a conditional handle in the graph being captured on `s` (for kernels that set it).
static int make_handle(cudaStream_t s, cudaGraphConditionalHandle* h, unsigned def) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t cg = nullptr;
  cudaError_t e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, nullptr, nullptr);
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(h, cg, def, cudaGraphCondAssignDefault);
  return e == cudaSuccess ? PGJ_OK : set_cuda_error(e);
}

// Captures `fn(stream)` into `body` on a private stream.
template <typename F>
static int capture_into(cudaGraph_t body, F&& fn) {
  cudaStream_t s2;
  cudaError_t e = cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking);
  if (e != cudaSuccess) return set_cuda_error(e);
  int st;
  e = cudaStreamBeginCaptureToGraph(s2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    st = set_cuda_error(e);
  } else {
    st = fn(s2);
    cudaGraph_t bg = body;
    cudaError_t e2 = cudaStreamEndCapture(s2, &bg);
    if (!st && e2 != cudaSuccess) st = set_cuda_error(e2);
  }
  cudaStreamDestroy(s2);
  return st;
}

// Mixed reliable-update iteration (FP32 recurrence, inner records active):
// operator, update, IF(any load flagged){x += d; r64 = f - K64 x; r = T(r64)}, Green, p update.
static int capture_iteration_rel(pgj_ctx* c, int L, cudaStream_t s, cudaGraphConditionalHandle hw) {
  int st;
  const bool fused = c->fused != 0;
  if ((st = launch_recurrence_operator(c, L, PGJ_FP32, s))) return st;
  if (fused) st = launch_fxy(c, L, PGJ_FP32, kSlabUpdateL, c->d, s);
  else st = launch_update_ur(c, L, PGJ_FP32, nullptr, c->d, s);
  if (st) return st;
  cudaGraphConditionalHandle hif = 0;
  if ((st = make_handle(s, &hif, 0))) return st;
  if ((st = launch_rel_cond(c, L, hif, s))) return st;
  cudaGraph_t ifbody = nullptr;
  if ((st = add_conditional(s, &hif, 0, cudaGraphCondTypeIf, &ifbody))) return st;
  st = capture_into(ifbody, [&](cudaStream_t s3) {
    int r = launch_rel_fold(c, L, false, s3);
    if (r) return r;
    LoadScalars* saved = c->scal;
    c->scal = c->scal_out;
    r = launch_stencil(c, kResidual, L, PGJ_FP64, c->x, c->r64, c->f, nullptr, s3, c->scal_in);
    c->scal = saved;
    if (r) return r;
    // flagged loads restart from T(r64); the fused form also re-transforms their residual
    return fused ? launch_fxy(c, L, PGJ_FP32, kSlabSyncL, nullptr, s3) : launch_rel_sync(c, L, s3);
  });
  if (st) return st;
  if (fused) {
    if ((st = launch_fz_fused(c, L, PGJ_FP32, false, s))) return st;
    return launch_ifxy(c, L, PGJ_FP32, false, s, hw, true);
  }
  if ((st = launch_green(c, L, PGJ_FP32, c->r, false, s))) return st;
  return launch_update_p(c, L, PGJ_FP32, false, s, hw, true);
}

static int end_capture(cudaStream_t s, cudaGraph_t* g, int st) {
  cudaError_t e = cudaStreamEndCapture(s, g);
  if (st) { if (*g) cudaGraphDestroy(*g); *g = nullptr; return st; }
  if (e != cudaSuccess) return set_cuda_error(e);
  return PGJ_OK;
}

// Appends to the capture on `s`: directions init, then WHILE(any load active){iteration}.
static int capture_pcg(pgj_ctx* c, int L, cudaStream_t s, bool reliable = false) {
  int st = capture_first_direction(c, L, s);
  if (st) return st;
  cudaStreamCaptureStatus cs;
  cudaGraph_t cg = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  cudaError_t e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &ndeps);
  cudaGraphConditionalHandle h = 0;
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, cg, 1, cudaGraphCondAssignDefault);
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node = nullptr;
  if (e == cudaSuccess) e = cudaGraphAddNode(&node, cg, deps, ndeps, &cp);
  if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies);
  if (e != cudaSuccess) return set_cuda_error(e);
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  cudaStream_t s2;
  e = cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking);
  if (e != cudaSuccess) return set_cuda_error(e);
  e = cudaStreamBeginCaptureToGraph(s2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    st = set_cuda_error(e);
  } else {
    st = reliable ? capture_iteration_rel(c, L, s2, h) : capture_iteration(c, L, s2, h, true);
    cudaGraph_t bg = body;
    cudaError_t e2 = cudaStreamEndCapture(s2, &bg);
    if (!st && e2 != cudaSuccess) st = set_cuda_error(e2);
  }
  cudaStreamDestroy(s2);
  return st;
}

// One attempt: FP64 -> init masks, PCG loop, certify; mixed reliable -> FP32 recurrence with
// true-residual replacements, fold, certify; mixed sweeps -> one refinement sweep.
static int capture_attempt(pgj_ctx* c, int L, cudaStream_t s) {
  int st;
  if (c->prec == PGJ_FP32 && c->mixed_mode == 0) {
    st = launch_rel_start(c, L, s);
    if (!st) {
      c->scal = c->scal_in;
      st = capture_pcg(c, L, s, true);
      c->scal = c->scal_out;
    }
    if (!st) st = launch_rel_fold(c, L, true, s);
  } else if (c->prec == PGJ_FP32) {
    st = launch_inner_start(c, L, c->inner_rtol, s);
    if (!st) {
      c->scal = c->scal_in;
      st = capture_pcg(c, L, s);
      c->scal = c->scal_out;
    }
    if (!st) st = launch_inner_finish(c, L, s);
  } else {
    st = launch_init_mask(c, L, s);
    if (!st) st = capture_pcg(c, L, s);
  }
  if (!st) st = capture_cert(c, L, s);
  return st;
}

// Whole certified solve as one graph (FP64 and mixed reliable-update modes):
// counters <- 0; f = rhs(macros); targets; certify; WHILE(restart){attempt; decide}.
static int build_solve_graph(pgj_ctx* c, int L, double rtol) {
  Graphs* G = c->graphs;
  if (G->solve && G->loads == L && G->rtol == rtol && G->mode == c->mixed_mode) return PGJ_OK;
  if (G->solve) { cudaGraphExecDestroy(G->solve); G->solve = nullptr; }
  cudaStream_t s = G->cap;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return set_cuda_error(e);
  int st = PGJ_OK;
  c->scal = c->scal_out;
  if ((e = cudaMemsetAsync(c->cond, 0, 8 * sizeof(int), s)) != cudaSuccess) st = set_cuda_error(e);
  if (!st) st = launch_rhs(c, L, c->macros, c->f, s);
  if (!st) st = launch_norms(c, L, c->f, rtol, s);
  if (!st) st = capture_cert(c, L, s);
  cudaGraphConditionalHandle h = 0;
  cudaGraph_t body = nullptr;
  if (!st) st = add_conditional(s, &h, 1, cudaGraphCondTypeWhile, &body);
  if (!st)
    st = capture_into(body, [&](cudaStream_t s2) {
      int r = capture_attempt(c, L, s2);
      return r ? r : launch_decide(c, L, h, s2);
    });
  if ((st = end_capture(s, &g, st))) return st;
  e = cudaGraphInstantiate(&G->solve, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return set_cuda_error(e);
  G->loads = L;
  G->rtol = rtol;
  G->mode = c->mixed_mode;
  return PGJ_OK;
}

static int build_graphs(pgj_ctx* c, int L) {
  Graphs* G = c->graphs;
  if (G->attempt_loads == L && G->cert && G->attempt && G->inner_rtol == c->inner_rtol &&
      G->attempt_mode == c->mixed_mode)
    return PGJ_OK;
  if (G->cert) { cudaGraphExecDestroy(G->cert); G->cert = nullptr; }
  if (G->attempt) { cudaGraphExecDestroy(G->attempt); G->attempt = nullptr; }
  cudaStream_t s = G->cap;
  cudaGraph_t g = nullptr;
  int st;
  cudaError_t e;
  // certification graph
  if ((e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return set_cuda_error(e);
  st = capture_cert(c, L, s);
  if ((st = end_capture(s, &g, st))) return st;
  e = cudaGraphInstantiate(&G->cert, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return set_cuda_error(e);
  // one attempt (see capture_attempt)
  if ((e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return set_cuda_error(e);
  st = capture_attempt(c, L, s);
  if ((st = end_capture(s, &g, st))) return st;
  e = cudaGraphInstantiate(&G->attempt, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return set_cuda_error(e);
  G->attempt_loads = L;
  G->attempt_mode = c->mixed_mode;
  G->inner_rtol = c->inner_rtol;
  return PGJ_OK;
}

}  // namespace pgj

using namespace pgj;

extern "C" {

int pgj_version(void) { return 1; }

const char* pgj_status_string(int status) {
  switch (status) {
    case PGJ_OK: return "ok";
    case PGJ_ERR_ARGUMENT: return "invalid argument (pointer, size, shape or value)";
    case PGJ_ERR_UNSUPPORTED:
      return "unsupported grid size (FFT radices 2,3,5, even n, 4 <= n <= 256) or option for this context";
    case PGJ_ERR_LAUNCH: return "CUDA launch or runtime error";
    case PGJ_ERR_NONFINITE: return "non-finite value or non-positive curvature";
    case PGJ_ERR_ITERATION_CAP: return "iteration cap reached without certification";
    case PGJ_ERR_CERTIFICATION: return "true residual certification failed";
    case PGJ_ERR_TIMEOUT: return "bounded device wait expired";
    case PGJ_ERR_WORKSPACE: return "workspace missing, too small or misaligned";
    default: return "unknown status";
  }
}

int pgj_last_cuda_error(void) { return g_last_cuda_error; }

static bool grid_ok(int n) {
  FFTPlan p;
  return n >= 4 && n <= 256 && make_fft_plan(n, &p);
}

static bool batch_ok(int designs, int loads, int precision) {
  return designs >= 1 && designs <= kMaxDesigns && loads >= 1 && loads <= kMaxLoads &&
         (precision == PGJ_FP64 || precision == PGJ_FP32);
}

int pgj_workspace_bytes_batch(int n, int designs, int loads, int precision, size_t* bytes) {
  if (!bytes || !batch_ok(designs, loads, precision)) return PGJ_ERR_ARGUMENT;
  if (!grid_ok(n)) return PGJ_ERR_UNSUPPORTED;
  *bytes = make_layout(n, designs, loads, precision).total;
  return PGJ_OK;
}

int pgj_workspace_bytes(int n, int loads, int precision, size_t* bytes) {
  return pgj_workspace_bytes_batch(n, 1, loads, precision, bytes);
}

int pgj_ctx_create_batch(int n, int designs, int loads, int precision, double lam, double mu, void* workspace,
                         size_t workspace_bytes, void* stream, pgj_ctx** out) {
  if (!out || !batch_ok(designs, loads, precision) || !(mu > 0) || !(lam + 2 * mu / 3 > 0)) return PGJ_ERR_ARGUMENT;
  if (!grid_ok(n)) return PGJ_ERR_UNSUPPORTED;
  Layout y = make_layout(n, designs, loads, precision);
  if (!workspace || workspace_bytes < y.total || (reinterpret_cast<uintptr_t>(workspace) & 255)) return PGJ_ERR_WORKSPACE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  pgj_ctx* c = new (std::nothrow) pgj_ctx();
  if (!c) return PGJ_ERR_ARGUMENT;
  c->n = n; c->D = designs; c->lpd = loads; c->L = designs * loads; c->prec = precision; c->lam = lam; c->mu = mu;
  c->N = (long long)n * n * n; c->ns = n / 2 + 1; c->Nh = (long long)n * n * c->ns;
  c->kc = make_opconst(n, lam, mu);
  make_fft_plan(n, &c->plan);
  c->sg = stencil_geom(n, loads);
  c->fg = fft_geom(n, precision == PGJ_FP32 ? 4 : 8, c->plan);
  c->lay = y;
  c->base = static_cast<char*>(workspace);
  c->bytes = workspace_bytes;
  char* b = c->base;
  c->a = reinterpret_cast<double*>(b + y.a);
  c->scale = reinterpret_cast<double*>(b + y.scale);
  c->symbol = reinterpret_cast<double*>(b + y.symbol);
  c->symbol32 = precision == PGJ_FP32 ? reinterpret_cast<float*>(b + y.symbol32) : nullptr;
  c->tw = b + y.tw;
  c->solutions = reinterpret_cast<double*>(b + y.solutions);
  c->f = reinterpret_cast<double*>(b + y.f);
  c->x = reinterpret_cast<double*>(b + y.x);
  c->r64 = precision == PGJ_FP32 ? reinterpret_cast<double*>(b + y.r64) : nullptr;
  c->r = b + y.r; c->p = b + y.p; c->q = b + y.q; c->sw = b + y.sw; c->spec = b + y.spec;
  c->qb = precision == PGJ_FP32 && n == 64 ? static_cast<void*>(b + y.qb) : nullptr;
  c->hg = hf_geom(n, loads);
  {
    // the halo-free operator pays off where the slab update's first-row pass is cheap: the n = 64
    // register-transform path (row tests by shifts); measured per size, every other grid was slower
    // per iteration with it (n = 16: 51.7 vs 47.6 us, 54: 263 vs 247, 96: 687 vs 683)
    const char* e = std::getenv("PGJ_HF");
    c->hf = c->qb != nullptr && !(e && e[0] == '0') ? 1 : 0;
  }
  c->shat = b + y.shat;
  c->scale32 = precision == PGJ_FP32 ? reinterpret_cast<float*>(b + y.scale32) : nullptr;
  c->partials = reinterpret_cast<double*>(b + y.partials);
  c->scal_out = reinterpret_cast<LoadScalars*>(b + y.scal);
  c->scal_in = c->scal_out + c->L;
  c->scal = c->scal_out;
  c->d = precision == PGJ_FP32 ? static_cast<void*>(b + y.d) : nullptr;
  c->macros = reinterpret_cast<double*>(b + y.macros);
  c->cond = reinterpret_cast<int*>(b + y.cond);
  c->aux = reinterpret_cast<double*>(b + y.aux);
  c->alpha = 0.0;
  for (int d = 0; d < kMaxDesigns; ++d) c->alphas[d] = 0.0;
  c->inner_rtol = 1e-5;
  c->rel_delta2 = precision == PGJ_FP32 ? 1e-2 : 0.0;
  c->mixed_mode = 0;
  c->cap = 4000;  // the reference's per-load iteration cap (resident.py)
  c->last_refinements = 0;
  c->graphs = new (std::nothrow) Graphs();
  int st = PGJ_OK;
  cudaError_t e = cudaMemsetAsync(workspace, 0, y.total, s);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->graphs->cap, cudaStreamNonBlocking);
  if (e != cudaSuccess) st = set_cuda_error(e);
  if (!st) st = prepare_stencil_kernels();
  if (!st) st = prepare_fft_kernels();
  if (!st) st = prepare_slab_kernels();
  c->fused = slab_fits(c) && !std::getenv("PGJ_UNFUSED") ? 1 : 0;
  if (!st) st = init_fft_tables(c, s);
  if (!st) st = build_symbol(n, lam, mu, c->symbol, c->symbol32, s);
  if (!st) {
    // unit Voigt macros for the homogenized tensor
    double eye[36] = {0};
    for (int i = 0; i < 6; ++i) eye[i * 6 + i] = 1.0;
    e = cudaMemcpyAsync(c->aux + kAuxVoigt, eye, sizeof(eye), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = set_cuda_error(e);
  }
  if (!st) st = launch_scale(c, 0.5, s);  // stages the diagonal constants (once)
  for (int d = 0; d < designs && !st; ++d) {
    DesignScope view(c, d);
    st = launch_scale(c, 0.0, s);  // scale = 1 until an alpha is selected
  }
  if (!st) st = autotune_stencil(c, s);
  if (!st) st = autotune_fft(c, s);
  if (st) {
    delete c->graphs;
    delete c;
    return st;
  }
  *out = c;
  return PGJ_OK;
}

int pgj_ctx_create(int n, int loads, int precision, double lam, double mu, void* workspace, size_t workspace_bytes,
                   void* stream, pgj_ctx** out) {
  return pgj_ctx_create_batch(n, 1, loads, precision, lam, mu, workspace, workspace_bytes, stream, out);
}

int pgj_ctx_designs(pgj_ctx* ctx) { return ctx ? ctx->D : -1; }

int pgj_ctx_destroy(pgj_ctx* ctx) {
  if (!ctx) return PGJ_ERR_ARGUMENT;
  delete ctx->graphs;
  delete ctx;
  return PGJ_OK;
}

double* pgj_ctx_solutions(pgj_ctx* ctx) { return ctx ? ctx->solutions : nullptr; }
double* pgj_ctx_scale(pgj_ctx* ctx) { return ctx ? ctx->scale : nullptr; }
double* pgj_ctx_material(pgj_ctx* ctx) { return ctx ? ctx->a : nullptr; }

int pgj_set_material_at(pgj_ctx* c, int design, const double* a, void* stream) {
  if (!c || !a || design < 0 || design >= c->D) return PGJ_ERR_ARGUMENT;
  cudaError_t e = cudaMemcpyAsync(c->a + size_t(design) * size_t(c->N), a, sizeof(double) * size_t(c->N),
                                  cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? PGJ_OK : set_cuda_error(e);
}

int pgj_set_material(pgj_ctx* c, const double* a, void* stream) { return pgj_set_material_at(c, 0, a, stream); }

int pgj_set_alpha_at(pgj_ctx* c, int design, double alpha, void* stream) {
  if (!c || !std::isfinite(alpha) || design < 0 || design >= c->D) return PGJ_ERR_ARGUMENT;
  c->alphas[design] = alpha;
  if (design == 0) c->alpha = alpha;
  DesignScope view(c, design);
  return launch_scale(c, alpha, static_cast<cudaStream_t>(stream));
}

int pgj_set_alpha(pgj_ctx* c, double alpha, void* stream) { return pgj_set_alpha_at(c, 0, alpha, stream); }

int pgj_apply(pgj_ctx* c, int loads, const double* p, const int32_t* active, double* q, void* stream) {
  if (!c || !p || !q || loads < 1 || loads > c->L) return PGJ_ERR_ARGUMENT;
  return launch_stencil(c, kPlain, loads, PGJ_FP64, p, q, nullptr, active, static_cast<cudaStream_t>(stream));
}

int pgj_apply_f32(pgj_ctx* c, int loads, const float* p, const int32_t* active, float* q, void* stream) {
  if (!c || !p || !q || loads < 1 || loads > c->L) return PGJ_ERR_ARGUMENT;
  return launch_stencil(c, kPlain, loads, PGJ_FP32, p, q, nullptr, active, static_cast<cudaStream_t>(stream));
}

// Copies the (loads, 6) macro strains to the device unless the same values are already there
// (a pageable host-to-device copy serialises the stream, so repeated solves skip it).
static int stage_macros(pgj_ctx* c, int loads, const double* macros, cudaStream_t s) {
  for (int i = 0; i < 6 * loads; ++i)
    if (!std::isfinite(macros[i])) return PGJ_ERR_NONFINITE;
  if (c->staged_loads >= loads && std::memcmp(c->staged_macros, macros, sizeof(double) * 6 * size_t(loads)) == 0)
    return PGJ_OK;
  cudaError_t e = cudaMemcpyAsync(c->macros, macros, sizeof(double) * 6 * size_t(loads), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return set_cuda_error(e);
  std::memcpy(c->staged_macros, macros, sizeof(double) * 6 * size_t(loads));
  c->staged_loads = loads;
  return PGJ_OK;
}

int pgj_rhs(pgj_ctx* c, int loads, const double* macros, double* f, void* stream) {
  if (!c || !macros || !f || loads < 1 || loads > c->L) return PGJ_ERR_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int st = stage_macros(c, loads, macros, s);
  if (st) return st;
  return launch_rhs(c, loads, c->macros, f, s);
}

int pgj_precondition(pgj_ctx* c, int loads, const double* r, double* z, void* stream) {
  if (!c || !r || !z || loads < 1 || loads > c->L || c->prec != PGJ_FP64) return PGJ_ERR_ARGUMENT;
  return launch_green_standalone(c, loads, r, z, static_cast<cudaStream_t>(stream));
}

int pgj_green_symbol(int n, double lam, double mu, double* symbol, void* stream) {
  if (!symbol || !(mu > 0)) return PGJ_ERR_ARGUMENT;
  if (!grid_ok(n)) return PGJ_ERR_UNSUPPORTED;
  return build_symbol(n, lam, mu, symbol, nullptr, static_cast<cudaStream_t>(stream));
}

int pgj_set_inner_rtol(pgj_ctx* c, double inner_rtol) {
  if (!c || !(inner_rtol > 0 && inner_rtol < 1)) return PGJ_ERR_ARGUMENT;
  c->inner_rtol = inner_rtol;
  return PGJ_OK;
}

int pgj_last_refinements(pgj_ctx* c) { return c ? c->last_refinements : -1; }

int pgj_set_iteration_cap(pgj_ctx* c, int cap) {
  if (!c || cap < 1 || cap > 16000) return PGJ_ERR_ARGUMENT;
  c->cap = cap;
  c->graphs->loads = 0;  // the cap is a parameter of the captured kernels
  c->graphs->attempt_loads = 0;
  return PGJ_OK;
}

int pgj_iteration_cap(pgj_ctx* c) { return c ? c->cap : -1; }

int pgj_set_flexible_beta(pgj_ctx* c, int on) {
  if (!c || (on != 0 && on != 1)) return PGJ_ERR_ARGUMENT;
  if (on && c->prec != PGJ_FP32) return PGJ_ERR_UNSUPPORTED;
  c->flex = on;
  c->graphs->loads = 0;  // a parameter of the captured kernels
  c->graphs->attempt_loads = 0;
  return PGJ_OK;
}

int pgj_set_mixed_operator(pgj_ctx* c, int fp64) {
  if (!c || (fp64 != 0 && fp64 != 1)) return PGJ_ERR_ARGUMENT;
  if (c->prec != PGJ_FP32) return fp64 ? PGJ_OK : PGJ_ERR_UNSUPPORTED;  // FP64 contexts are FP64 throughout
  c->op64 = fp64;
  c->graphs->loads = 0;  // rebuild the solve graphs with the other operator
  c->graphs->attempt_loads = 0;
  return PGJ_OK;
}

int pgj_set_mixed_mode(pgj_ctx* c, int mode, double delta) {
  if (!c || (mode != 0 && mode != 1) || !(delta > 0 && delta < 1)) return PGJ_ERR_ARGUMENT;
  c->mixed_mode = mode;
  c->rel_delta2 = c->prec == PGJ_FP32 ? delta * delta : 0.0;
  c->graphs->loads = 0;  // rebuild the solve graphs with the new scheme
  c->graphs->attempt_loads = 0;
  return PGJ_OK;
}

// Maximum FP64 refinement sweeps of the mixed solve (each sweep: one FP32 inner PCG solve to
// inner_rtol relative, x += d, FP64 certification).
static constexpr int kMaxSweeps = 12;

int pgj_solve_async(pgj_ctx* c, int loads, const double* macros, double rtol, double* u, void* stream) {
  if (!c || !macros || !u || loads < 1 || loads > c->L || !(rtol > 0)) return PGJ_ERR_ARGUMENT;
  if (c->D > 1 && loads % c->lpd != 0) return PGJ_ERR_ARGUMENT;  // whole designs of a batched context
  if (c->prec == PGJ_FP32 && c->mixed_mode == 1) return PGJ_ERR_UNSUPPORTED;  // sweeps need the host
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t bytes = sizeof(double) * 3 * size_t(c->N) * loads;
  int st = stage_macros(c, loads, macros, s);
  if (!st) st = build_solve_graph(c, loads, rtol);
  if (st) return st;
  cudaError_t e = cudaSuccess;
  if (u != c->x) e = cudaMemcpyAsync(c->x, u, bytes, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = cudaGraphLaunch(c->graphs->solve, s);
  if (e == cudaSuccess && u != c->x) e = cudaMemcpyAsync(u, c->x, bytes, cudaMemcpyDeviceToDevice, s);
  if (e != cudaSuccess) return set_cuda_error(e);
  c->pending_loads = loads;
  return PGJ_OK;
}

int pgj_solve_wait(pgj_ctx* c, pgj_load_info* info, void* stream) {
  if (!c || !info || c->pending_loads < 1) return PGJ_ERR_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int loads = c->pending_loads;
  c->pending_loads = 0;
  std::vector<LoadScalars> h(loads);
  int cnt[8] = {0};
  cudaError_t e = cudaMemcpyAsync(h.data(), c->scal_out, sizeof(LoadScalars) * loads, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(cnt, c->cond, sizeof(cnt), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return set_cuda_error(e);
  bool all = true;
  for (int l = 0; l < loads; ++l) {
    pgj_load_info& I = info[l];
    const double thr = std::sqrt(h[l].target2);
    const bool ok = std::isfinite(h[l].absolute) && h[l].absolute <= thr && h[l].bad == 0;
    I.rhs_norm = h[l].norm;
    I.absolute_residual = h[l].absolute;
    I.threshold = thr;
    I.relative_residual = h[l].absolute / (h[l].norm > 1e-300 ? h[l].norm : 1e-300);
    I.iterations = h[l].iterations;
    I.converged = ok;
    I.restarts = h[l].restarts;
    I.bad = h[l].bad;
    all = all && ok;
  }
  const long long attempts = cnt[4] + 1;
  // loop body: operator, update, 5 Green passes, p update (fused: operator, fxy, fz, ifxy), plus the
  // IF-condition kernel of the reliable-update form; the first direction is 6 kernels (fused FP32:
  // 7, with the FP32 scale copy) after the mask / recurrence-start kernel
  const long long body = (c->fused ? 4 : 8) + (c->prec == PGJ_FP32 ? 1 : 0);
  const long long first = first_direction_launches(c);
  if (c->prec == PGJ_FP32)  // rel start, first direction, fold, certify, decide; 3 per replacement
    c->last_launches = 2 + 3 + attempts * (1 + first + 1 + 3 + 1) + body * cnt[5] + 3LL * cnt[3];
  else  // init mask, first direction, certify, decide
    c->last_launches = 2 + 3 + attempts * (1 + first + 3 + 1) + body * cnt[5];
  c->last_refinements = c->prec == PGJ_FP32 ? 1 + cnt[3] : 1;
  if (cnt[2]) return PGJ_ERR_TIMEOUT;
  if (cnt[1]) return PGJ_ERR_ITERATION_CAP;
  return all ? PGJ_OK : PGJ_ERR_CERTIFICATION;
}

int pgj_solve(pgj_ctx* c, int loads, const double* macros, double rtol, double* u, pgj_load_info* info, void* stream) {
  if (!c || !macros || !u || !info || loads < 1 || loads > c->L || !(rtol > 0)) return PGJ_ERR_ARGUMENT;
  if (c->D > 1 && c->prec == PGJ_FP32 && c->mixed_mode == 1) return PGJ_ERR_UNSUPPORTED;
  if (!(c->prec == PGJ_FP32 && c->mixed_mode == 1)) {
    const int st = pgj_solve_async(c, loads, macros, rtol, u, stream);
    return st ? st : pgj_solve_wait(c, info, stream);
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t N3 = 3 * size_t(c->N);
  const bool mixed = c->prec == PGJ_FP32 && c->mixed_mode == 1;  // restarted refinement sweeps
  c->scal = c->scal_out;
  int st = stage_macros(c, loads, macros, s);
  if (!st) st = launch_rhs(c, loads, c->macros, c->f, s);
  if (!st) st = launch_norms(c, loads, c->f, rtol, s);
  if (st) return st;
  cudaError_t e = cudaSuccess;
  if (u != c->x) e = cudaMemcpyAsync(c->x, u, sizeof(double) * N3 * loads, cudaMemcpyDeviceToDevice, s);
  if (e != cudaSuccess) return set_cuda_error(e);
  if ((st = build_graphs(c, loads))) return st;
  if ((e = cudaMemsetAsync(c->cond + 2, 0, sizeof(int), s)) != cudaSuccess) return set_cuda_error(e);
  if ((e = cudaGraphLaunch(c->graphs->cert, s)) != cudaSuccess) return set_cuda_error(e);
  std::vector<LoadScalars> h(loads);
  std::vector<int> ok(loads, 0);
  int restarts = 0, sweeps = 0;
  int body[4] = {0, 0, 0, 0};
  long long launches = 2 + 3;  // rhs + norms, initial certification
  bool capped_by_bound = false;
  auto read_state = [&](bool with_body) -> cudaError_t {
    cudaError_t err = cudaMemcpyAsync(h.data(), c->scal_out, sizeof(LoadScalars) * loads, cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess && with_body) err = cudaMemcpyAsync(body, c->cond, sizeof(body), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    return err;
  };
  auto evaluate = [&](bool& all, bool& anybad, bool& capped) {
    all = true; anybad = false; capped = false;
    for (int l = 0; l < loads; ++l) {
      const double thr = std::sqrt(h[l].target2);
      ok[l] = std::isfinite(h[l].absolute) && h[l].absolute <= thr && h[l].bad == 0;
      all = all && ok[l];
      anybad = anybad || h[l].bad;
      const int its = mixed ? h[l].total_iterations : h[l].iterations;
      capped = capped || (!ok[l] && its >= c->cap);
    }
  };
  if (mixed) {
    // one FP32 inner solve per sweep inside FP64 iterative refinement
    if ((e = read_state(false)) != cudaSuccess) return set_cuda_error(e);
    for (;;) {
      bool all, anybad, capped;
      evaluate(all, anybad, capped);
      if (all || anybad || capped || sweeps >= kMaxSweeps) break;
      if ((e = cudaGraphLaunch(c->graphs->attempt, s)) != cudaSuccess) return set_cuda_error(e);
      ++sweeps;
      if ((e = read_state(true)) != cudaSuccess) return set_cuda_error(e);
      // sweep: inner start + first direction, loop bodies, x += d, 3 certification kernels
      launches += 1 + first_direction_launches(c) + (c->fused ? 4LL : 8LL) * body[0] + 1 + 3;
      if (body[1]) { capped_by_bound = true; break; }
    }
  } else {
    for (;;) {
      if ((e = cudaGraphLaunch(c->graphs->attempt, s)) != cudaSuccess) return set_cuda_error(e);
      if ((e = read_state(true)) != cudaSuccess) return set_cuda_error(e);
      if (c->prec == PGJ_FP32)  // rel start + first direction, bodies, 3 per replacement, fold + certify
        launches += 1 + first_direction_launches(c) + (c->fused ? 5LL : 9LL) * body[0] + 3LL * body[3] + 1 + 3;
      else  // attempt: init mask + first direction, loop bodies, 3 certification kernels
        launches += 1 + first_direction_launches(c) + (c->fused ? 4LL : 8LL) * body[0] + 3;
      if (body[1]) { capped_by_bound = true; break; }
      bool all, anybad, capped;
      evaluate(all, anybad, capped);
      if (all || restarts >= 2 || anybad || capped) break;
      ++restarts;
    }
  }
  if (u != c->x) e = cudaMemcpyAsync(u, c->x, sizeof(double) * N3 * loads, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return set_cuda_error(e);
  bool all = true;
  for (int l = 0; l < loads; ++l) {
    pgj_load_info& I = info[l];
    const double thr = std::sqrt(h[l].target2);
    ok[l] = std::isfinite(h[l].absolute) && h[l].absolute <= thr && h[l].bad == 0;
    I.rhs_norm = h[l].norm;
    I.absolute_residual = h[l].absolute;
    I.threshold = thr;
    I.relative_residual = h[l].absolute / (h[l].norm > 1e-300 ? h[l].norm : 1e-300);
    I.iterations = mixed ? h[l].total_iterations : h[l].iterations;
    I.converged = ok[l];
    I.restarts = restarts;
    I.bad = h[l].bad;
    all = all && ok[l];
  }
  c->last_refinements = mixed ? sweeps : (c->prec == PGJ_FP32 ? 1 + body[3] : 1);
  c->last_launches = launches;
  if (body[2]) return PGJ_ERR_TIMEOUT;
  if (capped_by_bound) return PGJ_ERR_ITERATION_CAP;
  return all ? PGJ_OK : PGJ_ERR_CERTIFICATION;
}

long long pgj_last_launches(pgj_ctx* c) { return c ? c->last_launches : -1; }

int pgj_fused_iteration(pgj_ctx* c) { return c ? c->fused : -1; }

int pgj_tile_shapes(pgj_ctx* c, int* out) {
  if (!c || !out) return PGJ_ERR_ARGUMENT;
  out[0] = c->sg.ty; out[1] = c->sg.zc; out[2] = c->fg.rb; out[3] = c->fg.kcy; out[4] = c->fg.kcz;
  out[5] = c->fused;
  return PGJ_OK;
}

int pgj_tile_config(pgj_ctx* c, int* out) {
  if (!c || !out) return PGJ_ERR_ARGUMENT;
  out[0] = c->sg.ty; out[1] = c->sg.zc; out[2] = c->sg.stages; out[3] = c->sg.occ;
  out[4] = c->fft_req[0]; out[5] = c->fft_req[1]; out[6] = c->fft_req[2];
  out[7] = c->fused; out[8] = c->tile_source;
  return PGJ_OK;
}

int pgj_set_fused_iteration(pgj_ctx* c, int on) {
  if (!c || (on != 0 && on != 1)) return PGJ_ERR_ARGUMENT;
  if (on && !slab_fits(c)) return PGJ_ERR_UNSUPPORTED;
  c->fused = on;
  c->graphs->loads = 0;  // rebuild the solve graphs with the other kernel set
  c->graphs->attempt_loads = 0;
  return PGJ_OK;
}

int pgj_selftest_wait_timeout(pgj_ctx* c, int tries, void* stream) {
  if (!c || tries < 1) return PGJ_ERR_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(c->cond + 6, 0, sizeof(int), s);
  if (e != cudaSuccess) return set_cuda_error(e);
  int st = launch_wait_selftest(tries, c->cond + 6, s);
  if (st) return st;
  int flag = 0;
  e = cudaMemcpyAsync(&flag, c->cond + 6, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return set_cuda_error(e);
  return flag ? PGJ_ERR_TIMEOUT : PGJ_OK;
}

int pgj_profile_iteration(pgj_ctx* c, int loads, const double* macros, int reps, double* ms, double* bytes,
                          void* stream) {
  if (!c || !macros || !ms || !bytes || loads < 1 || loads > c->L || reps < 1) return PGJ_ERR_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t N = size_t(c->N), N3 = 3 * N, Nh = size_t(c->Nh);
  const int prec = c->prec;
  c->scal = c->scal_out;
  int st = stage_macros(c, loads, macros, s);
  if (!st) st = launch_rhs(c, loads, c->macros, c->f, s);
  if (!st) st = launch_norms(c, loads, c->f, 1e-30, s);  // tiny target: loads stay active while timed
  if (st) return st;
  cudaError_t e = cudaMemsetAsync(c->x, 0, sizeof(double) * N3 * loads, s);
  if (e != cudaSuccess) return set_cuda_error(e);
  if ((st = capture_cert(c, loads, s))) return st;
  if (prec == PGJ_FP32) {
    if ((st = launch_inner_start(c, loads, c->inner_rtol, s))) return st;
    c->scal = c->scal_in;
  } else if ((st = launch_init_mask(c, loads, s))) {
    return st;
  }
  if (!st) st = capture_first_direction(c, loads, s);
  const bool fused = c->fused != 0;
  void* u = prec == PGJ_FP32 ? c->d : static_cast<void*>(c->x);
  cudaEvent_t ev[2 * PGJ_PROFILE_KERNELS];
  for (int k = 0; k < 2 * PGJ_PROFILE_KERNELS; ++k) cudaEventCreate(&ev[k]);
  double acc[PGJ_PROFILE_KERNELS] = {0};
  auto launch_k = [&](int k) -> int {
    if (k == 0) return launch_recurrence_operator(c, loads, prec, s);
    if (fused && k == 1) return launch_fxy(c, loads, prec, kSlabUpdateL, u, s);
    if (fused && k == 2) return launch_fz_fused(c, loads, prec, false, s);
    if (fused && k == 3) return launch_ifxy(c, loads, prec, false, s, 0, false);
    if (fused) return PGJ_OK;
    if (k == 1) return prec == PGJ_FP32 ? launch_update_ur(c, loads, prec, nullptr, c->d, s)
                                        : launch_update_ur(c, loads, prec, c->x, nullptr, s);
    if (k < 7) return launch_green_pass(c, loads, prec, c->r, false, k - 2, s);
    return launch_update_p(c, loads, prec, false, s, 0, false);
  };
  // each kernel `reps` times back to back between its two events (after two warm launches), so the
  // device never waits for the host between them; the kernels run in iteration order. Repeating a
  // kernel re-applies its update to the same vectors, which changes values but not the work done.
  for (int k = 0; k < PGJ_PROFILE_KERNELS && !st; ++k) {
    for (int w = 0; w < 2 && !st; ++w) st = launch_k(k);
    cudaEventRecord(ev[2 * k], s);
    for (int rep = 0; rep < reps && !st; ++rep) st = launch_k(k);
    cudaEventRecord(ev[2 * k + 1], s);
  }
  if (!st && (e = cudaStreamSynchronize(s)) != cudaSuccess) st = set_cuda_error(e);
  for (int k = 0; k < PGJ_PROFILE_KERNELS && !st; ++k) {
    float t = 0.f;
    cudaEventElapsedTime(&t, ev[2 * k], ev[2 * k + 1]);
    acc[k] = t;
  }
  c->scal = c->scal_out;
  for (int k = 0; k < 2 * PGJ_PROFILE_KERNELS; ++k) cudaEventDestroy(ev[k]);
  if (st) return st;
  const double sz = prec == PGJ_FP32 ? 4.0 : 8.0;     // bytes per real of the inner precision
  const double V = double(N3) * sz * loads;           // one DOF vector over all loads
  const double S = double(Nh) * 3 * 2 * sz * loads;  // one complex half spectrum over all loads
  // scale field: FP64, or the FP32 planar copy the fused FP32 slab kernels read
  const double sc = double(N3) * ((fused && prec == PGJ_FP32) ? 4.0 : 8.0);
  const double ub = prec == PGJ_FP32 ? V : 2 * V;   // iterate: FP64 x or the inner-precision correction
  const double fused_algo[PGJ_PROFILE_KERNELS] = {
      2 * V + 8.0 * N,                            // operator: read p (+a), write q
      4 * V + ub + sc + S,                        // fxy: read p q r (+u +s), write r (+u), write spectrum
      2 * S + 6.0 * Nh * sz + S / loads,          // fz: spectrum in/out, symbol, DFT(s)
      S + sc + 2 * V, 0, 0, 0, 0};                // ifxy: read spectrum (+s) and p, write p
  const double algo[PGJ_PROFILE_KERNELS] = {
      2 * V + 8.0 * N,                  // operator: read p (+a), write q
      6 * V,                            // update_ur: read u p r q, write u r
      V + sc + S,                       // fft_x: read r (+s), write spectrum
      2 * S,                            // fft_y
      2 * S + 6.0 * Nh * sz,            // fft_z: spectrum in/out + symbol
      2 * S,                            // ifft_y
      S + sc + V,                       // ifft_x: read spectrum (+s), write s.w
      3 * V};                           // update_p: read s.w p, write p
  for (int k = 0; k < PGJ_PROFILE_KERNELS; ++k) {
    ms[k] = acc[k] / reps;
    bytes[k] = fused ? fused_algo[k] : algo[k];
  }
  return PGJ_OK;
}

int pgj_energies(pgj_ctx* c, int loads, const double* u, const double* macros, double* e, void* stream) {
  if (!c || !u || !macros || !e || loads < 1 || loads > kMaxLoads || loads > c->L) return PGJ_ERR_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int st = stage_macros(c, loads, macros, s);
  if (st) return st;
  return launch_energies(c, loads, u, c->macros, e, s);
}

int pgj_effective_tensor_at(pgj_ctx* c, int design, const double* u, double* C, void* stream) {
  if (!c || !u || !C || design < 0 || design >= c->D) return PGJ_ERR_ARGUMENT;
  return launch_effective_tensor(c, c->a + size_t(design) * size_t(c->N), u, C, nullptr,
                                 static_cast<cudaStream_t>(stream));
}

int pgj_effective_tensor(pgj_ctx* c, const double* u, double* C, void* stream) {
  return pgj_effective_tensor_at(c, 0, u, C, stream);
}

}  // extern "C"
