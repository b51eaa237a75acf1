// FP64 kernels of the FR residual-and-update path (plain form).
//
// One CTA owns one element ("cell") and gathers every correction that lands on
// it in ascending face-color order, so the sum order per cell is the order in
// which the reference's colored Numba kernels scatter into that cell
// (core/fr_residual/inviscid_kernel_colored.py:43-236,
// core/fr_residual/viscous_flux_kernel.py:292-520): no atomics, bit-stable
// results run to run.
//
// Template dims: S solution points, FN over-integration points, NP flux points
// per face, N1D points per direction.
#pragma once
#include "afr_device.cuh"

namespace afr {

struct StageArgs {
  const double* Ucur;   // state the residual is evaluated on (N,S,nv)
  const double* U0;     // step-start state (RK combination)
  const double* U1;     // stage-1 state (RK stage 2 combination)
  double* Unext;        // output state (N,S,nv)
  const double* grads;  // (N,S,12): du_a/dx_b (9), dT/dx_b (3), of Ucur
  const double* nut;    // (N,S) kinematic eddy viscosity or null
  const double* dt;     // (N,S)
  double* Rinv;         // residual-only mode outputs (N,S,nv), may be null
  double* Rvisc;
  double* norm_part;    // (N) per-cell sum of squares of dU/dt (stage 0)
  int nv;
  int stage;            // 0,1,2 RK stage, -1 residual only
  int inviscid_only;
  double mu;
  unsigned* status;
};

__device__ __forceinline__ int cell_type(const Geom& g, int e) { return e < g.n_prism ? 0 : 1; }

// out[r][c] (+)= sum_k A[r*lda + k] * B[k*ldb + c] for r<R, c<C; A global, B/out shared.
template <int R, int C, int K>
__device__ __forceinline__ void block_gemm(double* out, int ldo, const double* __restrict__ A, int lda,
                                           const double* B, int ldb) {
  for (int t = threadIdx.x; t < R * C; t += blockDim.x) {
    const int r = t / C, c = t % C;
    const double* a = A + (size_t)r * lda;
    double acc = 0.0;
#pragma unroll 4
    for (int k = 0; k < K; ++k) acc += __ldg(a + k) * B[k * ldb + c];
    out[r * ldo + c] = acc;
  }
}

// Median-based outlier zeroing over the S points of one cell, per variable
// (core/fr_operators/troubled_cell.py:346-408).  R is (S,5) in shared memory,
// Uref the cell's state rows (stride ldU, first 5 columns).  work >= 10 doubles.
template <int S>
__device__ void suppress_outliers(double* R, const double* Uref, int ldU, double* work) {
  double* med = work;       // [5]
  double* fmean = work + 5; // [5]
  // rank every |R[s,v]| among its column (stable), pick the middle one(s)
  for (int t = threadIdx.x; t < S * 5; t += blockDim.x) {
    const int s = t / 5, v = t % 5;
    const double x = fabs(R[s * 5 + v]);
    int rank = 0;
    for (int j = 0; j < S; ++j) {
      const double y = fabs(R[j * 5 + v]);
      rank += (y < x) || (y == x && j < s);
    }
    if (S & 1) {
      if (rank == S / 2) med[v] = x;
    } else {
      // even: average of ranks S/2-1 and S/2, combined below through two slots
      if (rank == S / 2 - 1) work[10 + v] = x;
      if (rank == S / 2) work[15 + v] = x;
    }
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    const int v = threadIdx.x;
    if (!(S & 1)) med[v] = 0.5 * (work[10 + v] + work[15 + v]);
    double acc = 0.0;
    for (int s = 0; s < S; ++s) acc += fabs(Uref[s * ldU + v]);
    fmean[v] = acc / S;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < S * 5; t += blockDim.x) {
    const int v = t % 5;
    const double ref = fmax(fmax(med[v], 1e-9 * fmean[v]), 1e-300);
    if (fabs(R[t]) > 1e4 * ref) R[t] = 0.0;
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// gradient pre-pass: grads of u,v,w,T at the S points of every cell
// (core/fr_operators/gradients.py:23-64 applied to Q and T as in
//  core/fr_residual/viscous_flux.py:161-166)
// ---------------------------------------------------------------------------
template <int S>
__global__ void __launch_bounds__(128) k_grad(Geom g, Ops ops, const double* __restrict__ U, int nv,
                                              double* __restrict__ grads) {
  __shared__ double f[S * 4];
  __shared__ double gc[S * 3 * 4];
  const int e = blockIdx.x;
  const int ct = cell_type(g, e);
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    double q[5];
    cons_to_prim(U + ((size_t)e * S + s) * nv, q);
    f[s * 4 + 0] = q[1];
    f[s * 4 + 1] = q[2];
    f[s * 4 + 2] = q[3];
    f[s * 4 + 3] = q[4] / (fmax(q[0], 1e-10) * R_AIR);
  }
  __syncthreads();
  block_gemm<S * 3, 4, S>(gc, 4, ops.D3g[ct], S, f, 4);
  __syncthreads();
  for (int t = threadIdx.x; t < S * 12; t += blockDim.x) {
    const int s = t / 12, c = t % 12;
    const int q = c / 3, n = c % 3;  // c = q*3+n: q in (u,v,w,T)
    const double* inv = g.inv + ((size_t)e * S + s) * 9;
    double acc = 0.0;
    for (int m = 0; m < 3; ++m) acc += gc[(s * 3 + m) * 4 + q] * inv[m * 3 + n];
    grads[((size_t)e * S + s) * 12 + c] = acc;
  }
}

// ---------------------------------------------------------------------------
// fused stage kernel: inviscid + viscous residual of one cell, outlier
// suppression, then (stage >= 0) the SSP-RK3 Shu-Osher combination,
// positivity projection and modal filter (core/time_integration/base.py:250-335,
// core/time_integration/positivity.py:13-45, core/fr_solver/filter.py:29-42).
// ---------------------------------------------------------------------------
template <int S, int FN, int NP>
struct StageSmem {
  static constexpr int NF = 18;  // Q(5) grads(12) mu_t(1) per point
  static constexpr int oU = 0;                      // S*8
  static constexpr int oQ = oU + S * 8;             // S*5
  static constexpr int oAdj = oQ + S * 5;           // S*9
  static constexpr int oG = oAdj + S * 9;           // S*13 (grads + mu_t)
  static constexpr int oRi = oG + S * 13;           // S*5
  static constexpr int oRv = oRi + S * 5;           // S*5
  static constexpr int oCi = oRv + S * 5;           // S*5
  static constexpr int oCv = oCi + S * 5;           // S*5
  static constexpr int oBig = oCv + S * 5;          // scratch shared by phases
  // volume phase scratch
  static constexpr int vQf = 0;                     // FN*5
  static constexpr int vFt = vQf + FN * 5;          // FN*15
  static constexpr int vDf = vFt + FN * 15;         // FN*5
  static constexpr int vEnd = vDf + FN * 5;
  // interface phase scratch
  static constexpr int iOwn = 0;                    // NP*21 : Q(5) arow(3) g(13)
  static constexpr int iOth = iOwn + NP * 21;       // NP*18 : Q(5) g(13)
  static constexpr int iNb = iOth + NP * 18;        // S*NF  neighbor fields
  static constexpr int iJi = iNb + S * NF;          // NP*5
  static constexpr int iJv = iJi + NP * 5;          // NP*5
  static constexpr int iEnd = iJv + NP * 5;
  static constexpr int big = vEnd > iEnd ? vEnd : iEnd;
  static constexpr int work = oBig + big;           // 20 doubles for reductions
  static constexpr int total = work + 24;
};

// load the 18 point fields of a neighbouring cell into shared memory
template <int S>
__device__ __forceinline__ void load_nb_fields(const StageArgs& a, int c, double* dst) {
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    const double* u = a.Ucur + ((size_t)c * S + s) * a.nv;
    double q[5];
    cons_to_prim(u, q);
    double* d = dst + s * 18;
    for (int v = 0; v < 5; ++v) d[v] = q[v];
    const double* gr = a.grads + ((size_t)c * S + s) * 12;
    for (int k = 0; k < 12; ++k) d[5 + k] = gr[k];
    d[17] = a.nut ? fmax(u[0], 1e-10) * a.nut[(size_t)c * S + s] : 0.0;
  }
}

template <int S, int FN, int NP, int N1D>
__global__ void __launch_bounds__(128) k_stage(Geom g, Ops ops, Faces fc, Bc bc, StageArgs a) {
  using L = StageSmem<S, FN, NP>;
  extern __shared__ double sm[];
  double* sU = sm + L::oU;
  double* sQ = sm + L::oQ;
  double* sAdj = sm + L::oAdj;
  double* sG = sm + L::oG;
  double* sRi = sm + L::oRi;
  double* sRv = sm + L::oRv;
  double* sCi = sm + L::oCi;
  double* sCv = sm + L::oCv;
  double* big = sm + L::oBig;
  double* work = sm + L::work;

  const int e = blockIdx.x;
  const int ct = cell_type(g, e);
  const int nv = a.nv;
  const bool visc = !a.inviscid_only;
  const double* det = g.det + (size_t)e * S;

  // ---- load own cell ----
  for (int t = threadIdx.x; t < S * nv; t += blockDim.x) sU[(t / nv) * 8 + t % nv] = a.Ucur[(size_t)e * S * nv + t];
  for (int t = threadIdx.x; t < S * 9; t += blockDim.x) sAdj[t] = g.adj[(size_t)e * S * 9 + t];
  __syncthreads();
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    double q[5];
    cons_to_prim(sU + s * 8, q);
    for (int v = 0; v < 5; ++v) sQ[s * 5 + v] = q[v];
    if (visc) {
      const double* gr = a.grads + ((size_t)e * S + s) * 12;
      for (int k = 0; k < 12; ++k) sG[s * 13 + k] = gr[k];
      sG[s * 13 + 12] = a.nut ? fmax(sU[s * 8], 1e-10) * a.nut[(size_t)e * S + s] : 0.0;
    }
  }
  for (int t = threadIdx.x; t < S * 5; t += blockDim.x) { sCi[t] = 0.0; sCv[t] = 0.0; }
  __syncthreads();

  // ---- inviscid volume term with over-integration (core/fr_residual/inviscid.py:186-266) ----
  {
    double* Qf = big + L::vQf;
    double* Ft = big + L::vFt;
    double* Df = big + L::vDf;
    block_gemm<FN, 5, S>(Qf, 5, ops.c2f[ct], S, sQ, 5);
    __syncthreads();
    for (int i = threadIdx.x; i < FN; i += blockDim.x) {
      double q[5], F[3][5];
      for (int v = 0; v < 5; ++v) q[v] = Qf[i * 5 + v];
      euler_flux(q, F);
      const double* ad = g.adj_fine + ((size_t)e * FN + i) * 9;
      double am[9];
      for (int k = 0; k < 9; ++k) am[k] = __ldg(ad + k);
      for (int m = 0; m < 3; ++m)
        for (int v = 0; v < 5; ++v)
          Ft[(i * 3 + m) * 5 + v] = am[m * 3 + 0] * F[0][v] + am[m * 3 + 1] * F[1][v] + am[m * 3 + 2] * F[2][v];
    }
    __syncthreads();
    block_gemm<FN, 5, FN * 3>(Df, 5, ops.Dfine[ct], FN * 3, Ft, 5);
    __syncthreads();
    block_gemm<S, 5, FN>(sRi, 5, ops.f2c[ct], FN, Df, 5);
    __syncthreads();
    for (int t = threadIdx.x; t < S * 5; t += blockDim.x) sRi[t] = -sRi[t] / det[t / 5];
  }

  // ---- viscous volume term (core/fr_residual/viscous_flux.py:178-207) ----
  if (visc) {
    double* Gt = big;  // S*15
    for (int s = threadIdx.x; s < S; s += blockDim.x) {
      double q[5], G[3][5];
      for (int v = 0; v < 5; ++v) q[v] = sQ[s * 5 + v];
      viscous_flux(q, sG + s * 13, sG + s * 13 + 9, a.mu, sG[s * 13 + 12], G);
      const double* am = sAdj + s * 9;
      for (int m = 0; m < 3; ++m)
        for (int v = 0; v < 5; ++v)
          Gt[(s * 3 + m) * 5 + v] = am[m * 3 + 0] * G[0][v] + am[m * 3 + 1] * G[1][v] + am[m * 3 + 2] * G[2][v];
    }
    __syncthreads();
    block_gemm<S, 5, S * 3>(sRv, 5, ops.D3[ct], S * 3, Gt, 5);
    __syncthreads();
    for (int t = threadIdx.x; t < S * 5; t += blockDim.x) sRv[t] = sRv[t] / det[t / 5];
  }
  __syncthreads();

  // ---- interface terms, gathered per cell in ascending color order ----
  double* own = big + L::iOwn;
  double* oth = big + L::iOth;
  double* nb = big + L::iNb;
  double* Ji = big + L::iJi;
  double* Jv = big + L::iJv;
  const int nown = visc ? 21 : 8;
  const int noth = visc ? 18 : 5;
  double vol_o = 0.0;
  if (visc) {
    for (int s = 0; s < S; ++s) vol_o += det[s];
    vol_o /= S;
  }
  const int s_beg = fc.slot_ptr[e], s_end = fc.slot_ptr[e + 1];
  for (int si = s_beg; si < s_end; ++si) {
    const int code = fc.slot[si];
    const int f = code >> 1;
    const bool is_owner = (code & 1) == 0;
    const int ax = is_owner ? fc.o_axis[f] : fc.n_axis[f];
    const double side = is_owner ? fc.o_side[f] : fc.n_side[f];
    const bool bnd = fc.is_bnd[f] != 0;
    const double* E = ops.extrap + (((size_t)ct * 3 + ax) * 2 + (side < 0.0 ? 0 : 1)) * NP * S;
    // own extrapolation: Q, adjugate row of this axis, grads+mu_t
    for (int t = threadIdx.x; t < NP * nown; t += blockDim.x) {
      const int i = t / nown, c = t % nown;
      const double* Er = E + i * S;
      double acc = 0.0;
      if (c < 5) {
        for (int s = 0; s < S; ++s) acc += __ldg(Er + s) * sQ[s * 5 + c];
      } else if (c < 8) {
        for (int s = 0; s < S; ++s) acc += __ldg(Er + s) * sAdj[s * 9 + ax * 3 + (c - 5)];
      } else {
        for (int s = 0; s < S; ++s) acc += __ldg(Er + s) * sG[s * 13 + (c - 8)];
      }
      own[i * 21 + c] = acc;
    }
    __syncthreads();
    // other side
    if (bnd) {
      for (int i = threadIdx.x; i < NP; i += blockDim.x) {
        double qo[5], n[3], gq[5];
        for (int v = 0; v < 5; ++v) qo[v] = own[i * 21 + v];
        const double* tn = fc.tnormal + ((size_t)f * NP + i) * 3;
        for (int d = 0; d < 3; ++d) n[d] = tn[d];
        ghost_state(bc, fc.bc_group[f], qo, n, gq);
        for (int v = 0; v < 5; ++v) oth[i * 18 + v] = gq[v];
        for (int k = 0; k < 13; ++k) oth[i * 18 + 5 + k] = own[i * 21 + 8 + k];
      }
    } else {
      const int c0 = is_owner ? fc.nb_c0[f] : fc.ow_c0[f];
      const int i1 = is_owner ? fc.nb_i1[f] : fc.ow_i1[f];
      for (int t = threadIdx.x; t < NP * 18; t += blockDim.x) oth[t] = 0.0;
      for (int src = 0; src < 2; ++src) {
        int c;
        const double* M;
        if (src == 0) {
          if (c0 < 0) continue;
          c = c0;
          M = (is_owner ? fc.nb_m0 : fc.ow_m0) + (size_t)f * NP * S;
        } else {
          if (i1 < 0) continue;
          c = is_owner ? fc.nb_c1[i1] : fc.ow_c1[i1];
          M = (is_owner ? fc.nb_m1 : fc.ow_m1) + (size_t)i1 * NP * S;
        }
        __syncthreads();
        load_nb_fields<S>(a, c, nb);
        __syncthreads();
        for (int t = threadIdx.x; t < NP * noth; t += blockDim.x) {
          const int i = t / noth, k = t % noth;
          const double* Mr = M + i * S;
          double acc = oth[i * 18 + k];
          for (int s = 0; s < S; ++s) {
            const double w = __ldg(Mr + s);
            if (w != 0.0) acc += w * nb[s * 18 + k];
          }
          oth[i * 18 + k] = acc;
        }
      }
    }
    __syncthreads();
    // pointwise fluxes at the NP flux points
    for (int i = threadIdx.x; i < NP; i += blockDim.x) {
      const double* ow = own + i * 21;
      const double* ot = oth + i * 18;
      const double a0 = ow[5], a1 = ow[6], a2 = ow[7];
      double mag = sqrt(a0 * a0 + a1 * a1 + a2 * a2);
      if (mag < 1e-300) mag = 1e-300;
      double dir[3] = {a0 / mag * side, a1 / mag * side, a2 / mag * side};
      const double* tn = fc.tnormal + ((size_t)f * NP + i) * 3;
      const double sg = is_owner ? 1.0 : -1.0;
      const double t0 = sg * tn[0], t1 = sg * tn[1], t2 = sg * tn[2];
      if (dir[0] * t0 + dir[1] * t1 + dir[2] * t2 < 0.5) { dir[0] = t0; dir[1] = t1; dir[2] = t2; }
      double qo[5], qn[5], Fc[5], Fp[3][5];
      for (int v = 0; v < 5; ++v) { qo[v] = ow[v]; qn[v] = ot[v]; }
      ausm_up(qo, qn, dir, Fc);
      euler_flux(qo, Fp);
      for (int v = 0; v < 5; ++v)
        Ji[i * 5 + v] = Fc[v] * mag * side - (a0 * Fp[0][v] + a1 * Fp[1][v] + a2 * Fp[2][v]);
      if (visc) {
        double qa[5], ga[13];
        for (int v = 0; v < 5; ++v) qa[v] = 0.5 * (qo[v] + qn[v]);
        for (int k = 0; k < 13; ++k) ga[k] = 0.5 * (ow[8 + k] + ot[5 + k]);
        double Gc[3][5], Go[3][5];
        viscous_flux(qa, ga, ga + 9, a.mu, ga[12], Gc);
        viscous_flux(qo, ow + 8, ow + 17, a.mu, ow[20], Go);
        double jv[5];
        for (int v = 0; v < 5; ++v)
          jv[v] = (a0 * Gc[0][v] + a1 * Gc[1][v] + a2 * Gc[2][v]) - (a0 * Go[0][v] + a1 * Go[1][v] + a2 * Go[2][v]);
        if (bnd) {
          // interior-penalty term on boundary faces (core/fr_operators/flux_kernels.py:140-200)
          double h = pow(vol_o, 1.0 / 3.0);
          if (h < 1e-300) h = 1e-300;
          const double eta = C_IP * (a.mu + ow[20]) / h;
          const double scale = eta * sqrt(a0 * a0 + a1 * a1 + a2 * a2) * side;
          for (int v = 1; v < 4; ++v) jv[v] += -scale * (qo[v] - qn[v]);
        }
        for (int v = 0; v < 5; ++v) Jv[i * 5 + v] = jv[v];
      }
    }
    __syncthreads();
    // lift to solution points with g'(coordinate) and accumulate
    const double* gp = side < 0.0 ? ops.g_left : ops.g_right;
    for (int t = threadIdx.x; t < S * 5; t += blockDim.x) {
      const int s = t / 5, v = t % 5;
      const int fp = ops.dist_fp[ax * S + s];
      const double gw = gp[ops.dist_co[ax * S + s]];
      sCi[t] += -(gw * Ji[fp * 5 + v]) / det[s];
      if (visc) sCv[t] += (gw * Jv[fp * 5 + v]) / det[s];
    }
    __syncthreads();
  }

  for (int t = threadIdx.x; t < S * 5; t += blockDim.x) {
    sRi[t] = sRi[t] + sCi[t];
    if (visc) sRv[t] = sRv[t] + sCv[t];
  }
  __syncthreads();
  suppress_outliers<S>(sRi, sU, 8, work);
  if (visc) suppress_outliers<S>(sRv, sU, 8, work);

  if (a.stage < 0) {
    for (int t = threadIdx.x; t < S * nv; t += blockDim.x) {
      const int s = t / nv, v = t % nv;
      if (a.Rinv) a.Rinv[(size_t)e * S * nv + t] = v < 5 ? sRi[s * 5 + v] : 0.0;
      if (a.Rvisc) a.Rvisc[(size_t)e * S * nv + t] = (v < 5 && visc) ? sRv[s * 5 + v] : 0.0;
    }
    return;
  }

  // ---- RK stage combination + positivity (per point) ----
  double* Up = sCi;  // reuse: (S, 8)
  // sCi/sCv are S*5 each and contiguous: S*10 >= S*8
  __syncthreads();
  double part = 0.0;
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    double L[8], un[8];
    for (int v = 0; v < nv; ++v) L[v] = v < 5 ? sRi[s * 5 + v] + (visc ? sRv[s * 5 + v] : 0.0) : 0.0;
    if (a.stage == 0)
      for (int v = 0; v < nv; ++v) part += L[v] * L[v];
    const double dts = a.dt[(size_t)e * S + s];
    const double* u0 = a.U0 + ((size_t)e * S + s) * nv;
    const double* uc = sU + s * 8;
    if (a.stage == 0) {
      for (int v = 0; v < nv; ++v) un[v] = u0[v] + dts * L[v];
    } else if (a.stage == 1) {
      for (int v = 0; v < nv; ++v) un[v] = (0.75 * u0[v] + 0.25 * uc[v]) + (0.25 * dts) * L[v];
    } else {
      // 1/3 U0 + 0 U1 + 2/3 U2 + 2/3 dt L; the 0*U1 term is dropped: it can only
      // turn a finite value into NaN where U1 is non-finite, and U2 (filtered
      // from U1) is then non-finite at the same cell already.
      for (int v = 0; v < nv; ++v) un[v] = (1.0 / 3.0 * u0[v] + 2.0 / 3.0 * uc[v]) + (2.0 / 3.0 * dts) * L[v];
    }
    // enforce_positivity (p_floor = 1)
    const double rho = fmax(un[0], 1e-6);
    un[0] = rho;
    double vel[3] = {un[1] / rho, un[2] / rho, un[3] / rho};
    const double vm = sqrt(vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
    if (vm > 1e4) {
      const double cf = 1e4 / vm;
      for (int d = 0; d < 3; ++d) { vel[d] *= cf; un[1 + d] = rho * vel[d]; }
    }
    const double ke = 0.5 * rho * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
    const double p = (GAMMA - 1.0) * (un[4] - ke);
    if (p < 1.0) un[4] = 1.0 / (GAMMA - 1.0) + ke;
    if (nv > 5) un[5] = fmax(un[5], 0.0);
    if (nv > 6) un[6] = fmax(un[6], 1e-8);
    for (int v = 0; v < nv; ++v) Up[s * 8 + v] = un[v];
  }
  __syncthreads();
  // modal filter on the first five variables
  const double* Fm = ops.filt[ct];
  for (int t = threadIdx.x; t < S * nv; t += blockDim.x) {
    const int s = t / nv, v = t % nv;
    double val;
    if (v < 5) {
      double acc = 0.0;
      for (int j = 0; j < S; ++j) acc += __ldg(Fm + s * S + j) * Up[j * 8 + v];
      val = acc;
    } else {
      val = Up[s * 8 + v];
    }
    a.Unext[(size_t)e * S * nv + t] = val;
  }
  if (a.stage == 0) {
    // deterministic per-cell partial of sum(dU/dt^2)
    for (int off = 16; off > 0; off >>= 1) part += __shfl_down_sync(0xffffffffu, part, off);
    if ((threadIdx.x & 31) == 0) work[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
      double acc = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) acc += work[w];
      a.norm_part[e] = acc;
    }
  }
}

}  // namespace afr
