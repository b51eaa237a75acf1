// Kernels of the dual-time and IMEX integrators (the residuals themselves are
// the stage kernels of either arithmetic form, evaluated at arbitrary states).
// Restates (paths relative to the reference's src/autoflowcfd):
//   step_dual_time      core/time_integration/dual.py:19-158
//   step_imex           core/time_integration/imex.py:17-97
//   _ssp_rk_stage_step  core/time_integration/base.py:250-335
//   enforce_positivity  core/time_integration/positivity.py:13-45
//   _filter_flat_U      core/fr_solver/filter.py:29-42
// All arithmetic is FP64 in the order the reference's numpy expressions take.
#pragma once
#include "afr_kernels.cuh"

namespace afr {

// enforce_positivity with p_floor = 1 on one point's conserved values
__device__ __forceinline__ void positivity_point(double* un, int nv) {
  const double rho = fmax(un[0], 1e-6);
  un[0] = rho;
  double vel[3] = {un[1] / rho, un[2] / rho, un[3] / rho};
  const double vm = sqrt(vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
  if (vm > 1e4) {
    const double cf = 1e4 / vm;
    for (int d = 0; d < 3; ++d) {
      vel[d] *= cf;
      un[1 + d] = rho * vel[d];
    }
  }
  const double ke = 0.5 * rho * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
  const double pr = (GAMMA - 1.0) * (un[4] - ke);
  if (pr < 1.0) un[4] = 1.0 / (GAMMA - 1.0) + ke;
  if (nv > 5) un[5] = fmax(un[5], 0.0);
  if (nv > 6) un[6] = fmax(un[6], 1e-8);
}

// residual of the mean flow in the reference's R convention (dU/dt = -R):
// spatial R = -(inviscid + viscous), plus the BDF time derivative of the
// dual-time scheme (BDF1 without a previous level, BDF2 with one)
__device__ __forceinline__ double dual_residual(double rinv, double rvisc, double u, double un, const double* up,
                                                size_t i, double dtp) {
  const double rs = -(rinv + rvisc);
  if (!up) return rs + (u - un) / dtp;
  return rs + (3.0 * u - 4.0 * un + up[i]) / (2.0 * dtp);
}

struct ImpArgs {
  int64_t npts;           // cells * n_sps
  int nv;
  const double* U0;       // stage-0 state of the pseudo step (dual) / -
  const double* Ucur;     // the state the residuals below belong to
  const double* Rinv;     // inviscid residual (dU/dt) of Ucur (dual); of U^n (IMEX)
  const double* Rvisc;    // viscous residual (dU/dt) of Ucur
  const double* Un;       // dual: state at physical level n
  const double* Uprev;    // dual: state at level n-1, or nullptr (BDF1)
  double dtphys;          // dual: physical time step
  const double* dtl;      // local (pseudo) time step per point
  double scale;           // dual: CFL factor of the pseudo step; IMEX: damping factor
  int stage;              // dual: SSP-RK3 stage 0, 1, 2
  double* Unext;
};

// one SSP-RK3 stage of the pseudo-time iteration on the dual residual, with
// positivity; L = -R_dual(Ucur), dt = pseudo dt * CFL factor
__global__ void k_dual_stage(ImpArgs a) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.npts) return;
  const int nv = a.nv;
  const double dt = a.dtl[p] * a.scale;
  double un[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    if (v >= nv) {
      un[v] = 0.0;
      continue;
    }
    const size_t i = (size_t)p * nv + v;
    const double L = -dual_residual(a.Rinv[i], a.Rvisc[i], a.Ucur[i], a.Un[i], a.Uprev, i, a.dtphys);
    if (a.stage == 0) un[v] = a.U0[i] + dt * L;
    else if (a.stage == 1) un[v] = (0.75 * a.U0[i] + 0.25 * a.Ucur[i]) + (0.25 * dt) * L;
    else un[v] = (1.0 / 3.0 * a.U0[i] + 2.0 / 3.0 * a.Ucur[i]) + (2.0 / 3.0 * dt) * L;
  }
  positivity_point(un, nv);
#pragma unroll
  for (int v = 0; v < 8; ++v)
    if (v < nv) a.Unext[(size_t)p * nv + v] = un[v];
}

// damped Picard update of the IMEX scheme with positivity:
// U_next = U - (dt * (R_exp + R_imp)) * damping, R_exp = -inviscid(U^n),
// R_imp = -viscous(U)
__global__ void k_imex_update(ImpArgs a) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.npts) return;
  const int nv = a.nv;
  const double dt = a.dtl[p];
  double un[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    if (v >= nv) {
      un[v] = 0.0;
      continue;
    }
    const size_t i = (size_t)p * nv + v;
    const double total = -a.Rinv[i] + -a.Rvisc[i];
    un[v] = a.Ucur[i] - dt * total * a.scale;
  }
  positivity_point(un, nv);
#pragma unroll
  for (int v = 0; v < 8; ++v)
    if (v < nv) a.Unext[(size_t)p * nv + v] = un[v];
}

// positivity alone, in place
__global__ void k_positivity(double* U, int64_t npts, int nv) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  double un[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) un[v] = v < nv ? U[(size_t)p * nv + v] : 0.0;
  positivity_point(un, nv);
#pragma unroll
  for (int v = 0; v < 8; ++v)
    if (v < nv) U[(size_t)p * nv + v] = un[v];
}

// modal filter of the first five variables of every cell, in place: one CTA
// per cell, each output summed over the cell's points in order
// (np.einsum("sj,cjv->csv") of core/fr_solver/filter.py:29-42)
template <int S>
__global__ void k_filter_cells(Geom g, Ops ops, double* U, int nv) {
  __shared__ double sm[S * 5];
  const int c = blockIdx.x;
  double* Uc = U + (size_t)c * S * nv;
  for (int t = threadIdx.x; t < S * 5; t += blockDim.x) sm[t] = Uc[(t / 5) * nv + t % 5];
  __syncthreads();
  const double* F = ops.filt[cell_type(g, c)];
  for (int t = threadIdx.x; t < S * 5; t += blockDim.x) {
    const int s = t / 5, v = t % 5;
    double acc = 0.0;
    for (int j = 0; j < S; ++j) acc += __ldg(F + s * S + j) * sm[j * 5 + v];
    Uc[s * nv + v] = acc;
  }
}

// sums of squares in chunks of IMP_CHUNK elements (one partial per CTA), of
//   mode 0: the dual residual of Ucur;  mode 1: Ucur - U0;
//   mode 2: the IMEX total -inviscid(U^n) + -viscous(Ucur);  mode 3: inviscid + viscous (dU/dt)
constexpr int IMP_CHUNK = 65536, IMP_THREADS = 256;
__global__ void __launch_bounds__(IMP_THREADS) k_imp_sumsq(ImpArgs a, int mode, double* part) {
  __shared__ double sh[IMP_THREADS];
  const size_t n = (size_t)a.npts * a.nv;
  const size_t b0 = (size_t)blockIdx.x * IMP_CHUNK, b1 = b0 + IMP_CHUNK < n ? b0 + IMP_CHUNK : n;
  double acc = 0.0;
  for (size_t i = b0 + threadIdx.x; i < b1; i += IMP_THREADS) {
    double x;
    if (mode == 0) x = dual_residual(a.Rinv[i], a.Rvisc[i], a.Ucur[i], a.Un[i], a.Uprev, i, a.dtphys);
    else if (mode == 1) x = a.Ucur[i] - a.U0[i];
    else if (mode == 2) x = -a.Rinv[i] + -a.Rvisc[i];
    else x = a.Rinv[i] + a.Rvisc[i];
    acc += x * x;
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = IMP_THREADS / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

}  // namespace afr
