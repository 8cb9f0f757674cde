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

int launch_effective_tensor(pgj_ctx* c, const double* u, double* C, double* e, cudaStream_t s) {
  EnergyArgs A = energy_args(c, 6, u, c->aux + kAuxVoigt);  // unit Voigt macros (6 x 6)
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
