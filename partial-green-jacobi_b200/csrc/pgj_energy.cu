// Element strain energies and the homogenized tensor.
//
// For v_l = u_l + A_l on an element (A_l the affine field of the macro strain), the element
// energy v_i^T Ke v_j equals sum_m Q_i[m] . P_j[m] in the modal basis (the Hadamard transform is
// orthogonal up to the same factor on both sides), with P_j the modal element action for a = 1.
// One pass over the elements therefore gives every pair (i <= j) at once:
//   e_l(el)  = v_l^T Ke v_l / h^3                      (energy.cu:7-24 in exp/asg_scenarios_20261105)
//   C_ij     = mean_el( a v_i^T Ke v_j ) / h^3          (polarisation in reproduction.py:166-176)
#include "pgj_internal.h"

namespace pgj {

struct EnergyArgs {
  int n, loads;
  const double* u;       // (loads, 3N)
  const double* macros;  // (loads, 6) device
  const double* a;       // (N)
  double* e;             // (loads, N) or null
  double* C;             // 36 or null (pairs mode)
  LoadScalars* scal;     // ticket owner (record 0)
  double* partials;      // 21 * kMaxPartials
  OpConst kc;            // a = 1 constants of C0
};

constexpr int kEnergyThreads = 64;

template <bool PAIRS>
__global__ void __launch_bounds__(kEnergyThreads) k_energy(const EnergyArgs A) {
  const int n = A.n, L = A.loads;
  const size_t N = size_t(n) * n * n;
  extern __shared__ double Qsm[];  // [loads][21][kEnergyThreads]
  __shared__ double red[21 * 32];
  const int t = threadIdx.x;
  double acc[21];
#pragma unroll
  for (int k = 0; k < 21; ++k) acc[k] = 0.0;
  const double h = 1.0 / n, invv = double(n) * n * n;
  // each thread only touches its own column of Qsm: no block synchronisation inside the loop
  for (size_t ee = size_t(blockIdx.x) * blockDim.x + t; ee < N; ee += size_t(gridDim.x) * blockDim.x) {
    const int x = int(ee % n), y = int((ee / n) % n), z = int(ee / (size_t(n) * n));
    const double ae = A.a[ee];
    for (int l = 0; l < L; ++l) {
      const double* m = A.macros + 6 * l;
      // symmetric strain tensor of the engineering Voigt vector
      const double E[3][3] = {{m[0], m[5] / 2, m[4] / 2}, {m[5] / 2, m[1], m[3] / 2}, {m[4] / 2, m[3] / 2, m[2]}};
      double v[8][3];
      const double* ul = A.u + size_t(l) * 3 * N;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const int bx = b & 1, by = (b >> 1) & 1, bz = (b >> 2) & 1;
        const size_t node = (size_t(wrapi(z + bz, n)) * n + wrapi(y + by, n)) * n + wrapi(x + bx, n);
#pragma unroll
        for (int c = 0; c < 3; ++c)
          v[b][c] = ul[3 * node + c] + (E[c][0] * bx + E[c][1] * by + E[c][2] * bz) * h;
      }
      double Q[8][3];
      hadamard8<double>(v, Q);
#pragma unroll
      for (int mm = 1; mm < 8; ++mm)
#pragma unroll
        for (int c = 0; c < 3; ++c) Qsm[(size_t(l) * 21 + (mm - 1) * 3 + c) * kEnergyThreads + t] = Q[mm][c];
      if (!PAIRS || A.e) {
        double P[8][3];
        element_modal<double>(Q, 1.0, A.kc, P);
        double s = 0.0;
#pragma unroll
        for (int mm = 1; mm < 8; ++mm)
#pragma unroll
          for (int c = 0; c < 3; ++c) s += Q[mm][c] * P[mm][c];
        if (A.e) A.e[size_t(l) * N + ee] = s * invv;
      }
    }
    if (PAIRS) {
      int k = 0;
      for (int j = 0; j < L; ++j) {
        double Qj[8][3], Pj[8][3];
#pragma unroll
        for (int c = 0; c < 3; ++c) Qj[0][c] = 0.0;
#pragma unroll
        for (int mm = 1; mm < 8; ++mm)
#pragma unroll
          for (int c = 0; c < 3; ++c) Qj[mm][c] = Qsm[(size_t(j) * 21 + (mm - 1) * 3 + c) * kEnergyThreads + t];
        element_modal<double>(Qj, 1.0, A.kc, Pj);
        for (int i = 0; i <= j; ++i, ++k) {
          double s = 0.0;
#pragma unroll
          for (int mm = 1; mm < 8; ++mm)
#pragma unroll
            for (int c = 0; c < 3; ++c) s += Qsm[(size_t(i) * 21 + (mm - 1) * 3 + c) * kEnergyThreads + t] * Pj[mm][c];
          if (k < 21) acc[k] += ae * s;
        }
      }
    }
  }
  if constexpr (!PAIRS) {
    return;
  } else {
  // block reduction of the 21 pair sums
#pragma unroll
  for (int k = 0; k < 21; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_down_sync(0xffffffffu, acc[k], o);
  const int warp = t >> 5, lane = t & 31;
  if (lane == 0)
    for (int k = 0; k < 21; ++k) red[k * 32 + warp] = acc[k];
  __syncthreads();
  if (t < 21) {
    double s = 0.0;
    for (int w = 0; w < kEnergyThreads / 32; ++w) s += red[t * 32 + w];
    A.partials[size_t(t) * kMaxPartials + blockIdx.x] = s;
  }
  if (!last_block(&A.scal[0].ticket[kTicketAux2], gridDim.x)) return;
  if (t < 32) {
    for (int k = 0; k < 21; ++k) {
      const double s = warp_sum_partials(A.partials + size_t(k) * kMaxPartials, gridDim.x);
      if (t == 0) red[k] = s;
    }
    __syncwarp();
    if (t == 0) {
      int kk = 0;
      for (int j = 0; j < L; ++j)
        for (int i = 0; i <= j; ++i, ++kk) {
          const double v = red[kk] * invv / double(N);
          A.C[i * 6 + j] = v;
          A.C[j * 6 + i] = v;
        }
    }
  }
  }
}

static EnergyArgs energy_args(pgj_ctx* c, int loads, const double* u, const double* macros_dev) {
  EnergyArgs A;
  A.n = c->n; A.loads = loads; A.u = u; A.macros = macros_dev; A.a = c->a;
  A.e = nullptr; A.C = nullptr; A.scal = c->scal; A.partials = c->partials;
  A.kc = make_opconst(c->n, c->lam, c->mu);
  return A;
}

int launch_energies(pgj_ctx* c, int loads, const double* u, const double* macros_dev, double* e, cudaStream_t s) {
  if (loads < 1 || loads > kMaxLoads) return PGJ_ERR_ARGUMENT;
  EnergyArgs A = energy_args(c, loads, u, macros_dev);
  A.e = e;
  const unsigned blocks = unsigned((c->N + kEnergyThreads - 1) / kEnergyThreads);
  const size_t smem = size_t(loads) * 21 * kEnergyThreads * sizeof(double);
  cudaFuncSetAttribute(k_energy<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  k_energy<false><<<blocks, kEnergyThreads, smem, s>>>(A);
  return check_launch();
}

int launch_effective_tensor(pgj_ctx* c, const double* a, const double* u, double* C, double* e, cudaStream_t s) {
  EnergyArgs A = energy_args(c, 6, u, c->aux + kAuxVoigt);  // unit Voigt macros (6 x 6)
  A.a = a;
  A.C = C;
  A.e = e;
  unsigned blocks = 4 * 148;
  const unsigned need = unsigned((c->N + kEnergyThreads - 1) / kEnergyThreads);
  if (blocks > need) blocks = need;
  if (blocks > unsigned(kMaxPartials)) blocks = kMaxPartials;
  const size_t smem = size_t(6) * 21 * kEnergyThreads * sizeof(double);
  cudaFuncSetAttribute(k_energy<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  k_energy<true><<<blocks, kEnergyThreads, smem, s>>>(A);
  return check_launch();
}

}  // namespace pgj

// ------------------------------------------------------------------------------------------------
// Homogenized tensor without any device allocation by the caller or the library.
//
// Some callers cannot allocate device memory: a host application that owns the whole device
// memory pool and forbids third-party cudaMalloc (for instance a finite-element code that calls
// this library as a post-processing plugin inside its own memory budget). They still hold the
// density field and the six solutions, and want C_H from them. This entry point runs the same C_H
// kernel as pgj_effective_tensor, with its scratch (block partial sums and the last-block ticket)
// in a fixed file-scope device array instead of a context workspace; the six unit Voigt strains
// are a statically initialised device table, so nothing has to be copied before the first call.
//
// Limits and sharing: the array is kNoAllocScratchBytes (about 0.69 MB) on every GPU that loads
// the library, held until the process exits; it fits the kernel's partial sums for any grid the
// entry point accepts (2 <= n <= 256). Every call on a device uses the same array and the array
// keeps the last call's contents; the ticket is cleared at the start of each call. Two calls whose
// work overlaps on the GPU (for example on two streams without ordering) race on the array and
// give wrong results: order them on one stream or synchronise between them.
#include <mutex>

namespace {
constexpr size_t kNoAllocPartialDoubles = size_t(21) * pgj::kMaxPartials;
constexpr size_t kNoAllocScalarBytes = 256;
constexpr size_t kNoAllocScratchBytes = kNoAllocPartialDoubles * sizeof(double) + kNoAllocScalarBytes;
static_assert(sizeof(pgj::LoadScalars) <= kNoAllocScalarBytes, "scalar record must fit its slot");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
// (6, 6) unit engineering Voigt strains, one row per load
static __device__ const double g_noalloc_voigt[36] = {1, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0,
                                                      0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 1};

// Device addresses of the two symbols, looked up once per device with that device current and
// kept together with the id of the context they belong to: a replaced context (cudaDeviceReset,
// a new primary context) has another id, and the lookup is redone. The host-side names of the
// symbols are stand-ins, never passed to a kernel. A mutex orders first calls from several threads.
constexpr int kNoAllocMaxDevices = 64;
struct NoAllocSlot {
  unsigned long long ctx_id = 0;
  unsigned char* scratch = nullptr;
  const double* voigt = nullptr;
};
NoAllocSlot g_noalloc_slot[kNoAllocMaxDevices];
std::mutex g_noalloc_mutex;

// Current context id through the driver entry points the runtime exposes (no libcuda link).
// Returns 0 when the thread has no current context yet.
unsigned long long current_context_id() {
  using GetCurrent = int (*)(void**);
  using GetId = int (*)(void*, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
  });
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

int noalloc_setup(int device, unsigned char** scratch, const double** voigt) {
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  NoAllocSlot& slot = g_noalloc_slot[device];
  unsigned long long id = current_context_id();
  if (id != 0 && slot.ctx_id == id && slot.scratch) {
    *scratch = slot.scratch;
    *voigt = slot.voigt;
    return PGJ_OK;
  }
  void* p = nullptr;
  void* v = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e == cudaSuccess) e = cudaGetSymbolAddress(&v, g_noalloc_voigt);
  if (e != cudaSuccess) return pgj::set_cuda_error(e);
  if (id == 0) id = current_context_id();  // the lookup made the device's context current
  slot.ctx_id = id;
  slot.scratch = static_cast<unsigned char*>(p);
  slot.voigt = static_cast<const double*>(v);
  *scratch = slot.scratch;
  *voigt = slot.voigt;
  return PGJ_OK;
}
}  // namespace

extern "C" int pgj_effective_tensor_noalloc(int n, double lam, double mu, const double* a, const double* u,
                                            double* C, void* stream) {
  if (n < 2 || n > 256) return PGJ_ERR_ARGUMENT;  // beyond the grids this scratch is sized for
  if (!a || !u || !C || !(mu > 0) || !(lam + 2 * mu / 3 > 0)) return PGJ_ERR_ARGUMENT;
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return pgj::set_cuda_error(e);
  if (device < 0 || device >= kNoAllocMaxDevices) return PGJ_ERR_UNSUPPORTED;
  unsigned char* base = nullptr;
  const double* voigt = nullptr;
  int st = noalloc_setup(device, &base, &voigt);
  if (st) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* partials = reinterpret_cast<double*>(base);
  pgj::LoadScalars* scal = reinterpret_cast<pgj::LoadScalars*>(partials + kNoAllocPartialDoubles);
  // the last-block ticket must start at zero
  e = cudaMemsetAsync(scal, 0, sizeof(pgj::LoadScalars), s);
  if (e != cudaSuccess) return pgj::set_cuda_error(e);
  pgj::EnergyArgs A;
  A.n = n; A.loads = 6; A.u = u; A.macros = voigt; A.a = a;
  A.e = nullptr; A.C = C; A.scal = scal; A.partials = partials;
  A.kc = pgj::make_opconst(n, lam, mu);
  const size_t N = size_t(n) * n * n;
  unsigned blocks = 4 * 148;
  const unsigned need = unsigned((N + pgj::kEnergyThreads - 1) / pgj::kEnergyThreads);
  if (blocks > need) blocks = need;
  const size_t smem = size_t(6) * 21 * pgj::kEnergyThreads * sizeof(double);
  e = cudaFuncSetAttribute(pgj::k_energy<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return pgj::set_cuda_error(e);
  pgj::k_energy<true><<<blocks, pgj::kEnergyThreads, smem, s>>>(A);
  return pgj::check_launch();
}
