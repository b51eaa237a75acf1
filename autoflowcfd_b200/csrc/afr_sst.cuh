// SST k-omega source, transport and point-implicit update, and the local time
// step.  Restates (paths relative to the reference's src/autoflowcfd):
//   compute_turbulence_source          core/fr_solver/turbulence.py:178-330
//   SSTModelFR.compute_source_terms    core/turbulence/sst.py:241-354
//   SSTModelFR.update_fields           core/turbulence/sst.py:382-479
//   compute_turbulence_transport_residual core/turbulence/transport.py:367-522
//   transport face kernels             core/turbulence/transport_kernel.py:25-327
//   compute_local_time_step            core/fr_solver/cfl.py:12-147
#pragma once
#include "afr_kernels.cuh"

namespace afr {

struct SstArgs {
  const double* U;      // (N,S,nv) step-start state
  const double* dt;     // (N,S)
  double* k;            // (N,S) in/out
  double* w;            // (N,S) in/out
  double* nut;          // (N,S) in/out (kinematic eddy viscosity)
  double* pt;           // (N,S,5) scratch: Sk, Sw, beta_blend, gamma_k, gamma_w
  double* sp8;          // (N,S,8) scratch: rho, u, v, w, k, omega, gamma_k, gamma_w (face gathers)
  double* cfp;          // (F,P,4) scratch: conv_k, diff_k, conv_w, diff_w face corrections
  const uint8_t* wall_face;  // (F) WALL boundary faces (k Dirichlet-zero ghost)
  double* dbg;          // optional (N,S,4): Sk, Sw, transport_k, transport_w
  int nv;
  double mu;            // molecular viscosity of the mean flow
};

constexpr double SST_SK1 = 0.85, SST_SK2 = 1.0, SST_SW1 = 0.5, SST_SW2 = 0.856;
constexpr double SST_B1 = 0.075, SST_B2 = 0.0828, SST_A1 = 0.31, SST_KAPPA = 0.41, SST_BSTAR = 0.09;
constexpr double SST_TVR = 1.0e5;
constexpr double MU_SOURCE = 1.8e-5;  // hard-coded in core/fr_solver/turbulence.py:230

__device__ __forceinline__ double dfinite(double x) { return isfinite(x) ? x : 0.0; }

__device__ __forceinline__ double sst_F1(double k, double w, double d, double nu, double rho, double CD) {
  w = fmax(w, 1e-10);
  k = fmax(k, 1e-10);
  d = fmax(d, 1e-10);
  const double sk = sqrt(k);
  const double t1 = sk / (SST_BSTAR * w * d);
  const double t2 = 500.0 * nu / (d * d * w);
  const double t3 = 4.0 * rho * SST_SW2 * k / (fmax(CD, 1e-10) * (d * d));
  double a = fmin(fmax(t1, t2), t3);
  if (!isfinite(a)) a = 1e75;
  a = fmin(a, 1e75);
  const double a2 = a * a;
  return tanh(a2 * a2);  // arg1**4 (sst.py:92-141); within an ulp of pow(a, 4)
}

__device__ __forceinline__ double sst_F2(double k, double w, double d, double nu) {
  w = fmax(w, 1e-10);
  k = fmax(k, 1e-10);
  d = fmax(d, 1e-10);
  const double sk = sqrt(k);
  double a = fmax(2.0 * sk / (SST_BSTAR * w * d), 500.0 * nu / (d * d * w));
  if (!isfinite(a)) a = 1e150;
  a = fmin(a, 1e150);
  return tanh(a * a);
}

// SST cells per CTA (the three per-cell SST kernels)
template <int S>
struct SstTile {
  static constexpr int CPB = S <= 8 ? 8 : (S <= 27 ? 4 : 2);
  static constexpr int THREADS = 128;
};

// per cell: gradients of (rho u, rho v, rho w, k, omega), pointwise SST terms.
// CPB cells per CTA; cells [cell_base, cell_end) share one cell type.
template <int S>
__global__ void __launch_bounds__(128) k_sst_point(Geom g, Ops ops, SstArgs a, int cell_base, int cell_end) {
  constexpr int CPB = SstTile<S>::CPB;
  __shared__ double f[CPB * S * 5];     // rho u, rho v, rho w, k, omega; then the pt outputs
  __shared__ double gc[CPB * S * 3 * 5];
  __shared__ double sInv[CPB * S * 9];  // inverse Jacobians; then the sp8 outputs (row stride 9)
  __shared__ double sU[CPB * S * 7];    // state rows (stride nv = 7: SST handles carry n_vars 7)
  const int e0 = cell_base + blockIdx.x * CPB;
  const int nc = min(CPB, cell_end - e0);
  const int ct = cell_type(g, e0);
  const int nv = a.nv;
  // the tile's blocks are contiguous: asynchronous 8-byte copies, all in flight at once
  {
    const float rnv = 1.0f / float(nv);
    const double* ub = a.U + (size_t)e0 * S * nv;
    for (int t = threadIdx.x; t < nc * S * nv; t += blockDim.x) {
      cp_async8(sU + t, ub + t);
      const int p = __float2int_rz((float(t) + 0.5f) * rnv), v = t - p * nv;
      if (v >= 1 && v <= 3) cp_async8(f + p * 5 + v - 1, ub + t);
    }
    const double* ib = g.inv + (size_t)e0 * S * 9;
    for (int t = threadIdx.x; t < nc * S * 9; t += blockDim.x) cp_async8(sInv + t, ib + t);
    for (int t = threadIdx.x; t < nc * S; t += blockDim.x) {
      cp_async8(f + t * 5 + 3, a.k + (size_t)e0 * S + t);
      cp_async8(f + t * 5 + 4, a.w + (size_t)e0 * S + t);
    }
    cp_async_wait_all();
  }
  __syncthreads();
  // reference-space gradients (rows s*3+m of D3g) as one FP64 tensor-core
  // product: columns (cell, field)
  {
    dmma_product_rb<(5 * CPB + 7) / 8>(
        3 * S, 5 * nc, S, ops.fD3g[ct],
        [&](int j, int col) { return f[((col / 5) * S + j) * 5 + col % 5]; },
        [&](int r, int col, double x) { gc[((col / 5) * S * 3 + r) * 5 + col % 5] = x; });
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nc * S; t += blockDim.x) {
    const int s = t % S;
    const size_t p = (size_t)e0 * S + t;
    double inv[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) inv[k] = sInv[t * 9 + k];
    const double* gcs = gc + (size_t)(t - s) * 3 * 5;  // this cell's rows
    double gp[5][3];
    for (int q = 0; q < 5; ++q)
      for (int n = 0; n < 3; ++n) {
        double acc = 0.0;
        for (int m = 0; m < 3; ++m) acc += gcs[(s * 3 + m) * 5 + q] * inv[m * 3 + n];
        gp[q][n] = acc;
      }
    // |grad| <= 1e6 clip of grad k, grad omega
    for (int q = 3; q < 5; ++q) {
      const double mag = sqrt(gp[q][0] * gp[q][0] + gp[q][1] * gp[q][1] + gp[q][2] * gp[q][2]);
      if (mag > 1e6) {
        double sc = 1e6 / fmax(mag, 1e-10);
        sc = fmin(fmax(sc, 0.0), 1.0);
        for (int n = 0; n < 3; ++n) gp[q][n] *= sc;
      }
    }
    const double* u = sU + t * nv;
    const double rho = fmax(u[0], 1e-10);
    const double kf = f[t * 5 + 3], wf = f[t * 5 + 4];
    const double d = g.wall_dist[p];
    // strain magnitude of the conserved-momentum gradient
    double ss = 0.0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        const double sij = 0.5 * (gp[i][j] + gp[j][i]);
        ss += sij * sij;
      }
    const double Sm = sqrt(2.0 * ss);
    const double gd = gp[3][0] * gp[4][0] + gp[3][1] * gp[4][1] + gp[3][2] * gp[4][2];
    // --- compute_source_terms ---
    const double rrho = 1.0 / fmax(rho, 1e-10);  // one reciprocal: each use within an ulp of a division
    const double nu = MU_SOURCE * rrho;
    const double k_s = fmin(kf, 1e40);
    const double w_s = fmax(fmin(wf, 1e40), 1e-10);
    const double CD = fmax(2.0 * rho * SST_SW2 / w_s * gd, 1e-10);
    const double F1 = sst_F1(k_s, w_s, d, nu, rho, CD);
    const double F2 = sst_F2(k_s, w_s, d, nu);
    const double beta = F1 * SST_B1 + (1.0 - F1) * SST_B2;
    double nut = SST_A1 * fmax(k_s, 1e-10) / fmax(SST_A1 * fmax(w_s, 1e-10), F2 * fmax(Sm, 1e-10));
    nut = fmin(nut, SST_TVR * MU_SOURCE * rrho);
    if (!isfinite(nut)) nut = 0.0;
    double Pk = nut * rho * (Sm * Sm);
    Pk = fmin(Pk, 10.0 * SST_BSTAR * rho * k_s * w_s);
    const double Dk = rho * SST_BSTAR * k_s * w_s;
    const double g1 = SST_B1 / SST_BSTAR - SST_SW1 * SST_KAPPA * SST_KAPPA / sqrt(SST_BSTAR);
    const double g2 = SST_B2 / SST_BSTAR - SST_SW2 * SST_KAPPA * SST_KAPPA / sqrt(SST_BSTAR);
    const double gam = F1 * g1 + (1.0 - F1) * g2;
    const double Pw = rho * gam * (Sm * Sm);
    const double Dw = rho * beta * (w_s * w_s);
    const double CDw = 2.0 * rho * (1.0 - F1) * SST_SW2 / w_s * gd;
    const double Sk = dfinite(Pk - Dk);
    const double Sw = dfinite(Pw - Dw + CDw);
    // --- transport diffusion coefficients (mu = molecular viscosity of the mean flow) ---
    const double nu_m = a.mu * rrho;
    const double CD2 = fmax(2.0 * rho * SST_SW2 / fmax(wf, 1e-10) * gd, 1e-10);
    const double F1t = sst_F1(kf, wf, d, nu_m, rho, CD2);
    const double sk = F1t * SST_SK1 + (1.0 - F1t) * SST_SK2;
    const double sw = F1t * SST_SW1 + (1.0 - F1t) * SST_SW2;
    const double rnut = rho * nut;
    a.nut[p] = nut;
    // outputs staged in this point's own rows (read above by this thread only),
    // then stored as contiguous blocks
    const double gk = a.mu + sk * rnut, gw = a.mu + sw * rnut;
    const double r1 = u[1] * rrho, r2 = u[2] * rrho, r3 = u[3] * rrho;
    double* o = f + t * 5;
    o[0] = Sk;
    o[1] = Sw;
    o[2] = beta;
    o[3] = gk;
    o[4] = gw;
    double* o8 = sInv + t * 9;
    o8[0] = rho;
    o8[1] = r1;
    o8[2] = r2;
    o8[3] = r3;
    o8[4] = kf;
    o8[5] = wf;
    o8[6] = gk;
    o8[7] = gw;
  }
  __syncthreads();
  double* pt = a.pt + (size_t)e0 * S * 5;
  for (int t = threadIdx.x; t < nc * S * 5; t += blockDim.x) pt[t] = f[t];
  double* p8 = a.sp8 + (size_t)e0 * S * 8;
  for (int t = threadIdx.x; t < nc * S * 8; t += blockDim.x) p8[t] = sInv[(t >> 3) * 9 + (t & 7)];
}

// per face flux point: upwind convection and BR1-style diffusion corrections.
// One warp per face.  The face-point values are small FP64 products on the
// tensor path (mma.sync m8n8k4 .f64): owner side (face points x S) x (S x 8
// packed point values), neighbour side per source cell (face points x S) x
// (S x k, omega, gamma_k, gamma_w); the second source is added to the first as
// in the reference.  Lanes 0..P-1 then form the corrections.
constexpr int SST_FACE_WARPS = 4;

template <int S, int NP>
__global__ void __launch_bounds__(32 * SST_FACE_WARPS, 16) k_sst_face(Geom g, Ops ops, Faces fc, SstArgs a) {
  constexpr int W = SST_FACE_WARPS, RW = 17;  // RW: po (8), pn of the first (4) and second (4) source, pad
  constexpr int MT = (NP + 7) / 8;            // row tiles of the face points
  __shared__ double sR[W][NP * RW];
  const int wi = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int f = blockIdx.x * W + wi;
  if (f >= fc.F) return;  // whole warps: only warp-level synchronisation below
  const int oc = fc.owner[f];
  const int c0 = fc.nb_c0[f], i1 = fc.nb_i1[f];
  const int c1 = i1 >= 0 ? fc.nb_c1[i1] : -1;
  const bool bnd = c0 < 0 && i1 < 0;
  double* R = sR[wi];
  {
    const int ct = cell_type(g, oc);
    const int ax = fc.o_axis[f];
    const double* Ef =
        ops.fextrap + (((size_t)ct * 3 + ax) * 2 + (fc.o_side[f] <= 0.0 ? 0 : 1)) * (MT * ((S + 3) / 4) * 32);
    const double* X = a.sp8 + (size_t)oc * S * 8;
    dmma_warp_rb_f<MT, 1, S>(
        NP, 8, Ef, [&](int s, int n) { return __ldg(X + s * 8 + n); },
        [&](int i, int n, double x) { R[i * RW + n] = x; });
  }
  if (!bnd) {
    for (int src = 0; src < 2; ++src) {
      const int c = src == 0 ? c0 : c1;
      if (c < 0) continue;
      const double* X = a.sp8 + (size_t)c * S * 8 + 4;
      const double* M = src == 0 ? fmat(fc.nb_m0, fc.nb_m0i, f, 0, NP, S) : fmat(fc.nb_m1, fc.nb_m1i, i1, 0, NP, S);
      dmma_warp_rb<MT, 1, S>(
          NP, 4, [&](int i, int s) { return __ldg(M + s * NP + i); }, [&](int s, int n) { return __ldg(X + s * 8 + n); },
          [&](int i, int n, double x) { R[i * RW + 8 + src * 4 + n] = x; });
    }
  }
  __syncwarp();
  for (int i = lane; i < NP; i += 32) {
    const double* r = R + i * RW;
    double po[8], pn[4];
#pragma unroll
    for (int c = 0; c < 8; ++c) po[c] = r[c];
    if (bnd) {
      const bool wz = a.wall_face[f] != 0;
      pn[0] = wz ? -po[4] : po[4];
      pn[1] = po[5];
      pn[2] = po[6];
      pn[3] = po[7];
    } else {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double p0 = c0 >= 0 ? r[8 + q] : 0.0;
        pn[q] = c1 >= 0 ? p0 + r[12 + q] : p0;
      }
    }
    const double* tn = fc.tnormal + ((size_t)f * NP + i) * 3;
    const double mflux = ((po[0] * po[1]) * tn[0] + (po[0] * po[2]) * tn[1]) + (po[0] * po[3]) * tn[2];
    double* o = a.cfp + ((size_t)f * NP + i) * 4;
    const double upk = mflux >= 0.0 ? po[4] : pn[0];
    const double upw = mflux >= 0.0 ? po[5] : pn[1];
    o[0] = mflux * (upk - po[4]);
    o[1] = (0.5 * (po[6] + pn[2])) * (0.5 * (po[4] + pn[0]) - po[4]);
    o[2] = mflux * (upw - po[5]);
    o[3] = (0.5 * (po[7] + pn[3])) * (0.5 * (po[5] + pn[1]) - po[5]);
  }
}

// per cell: volume transport terms, gather of the face corrections, outlier
// suppression and the point-implicit k / omega update.  CPB cells per CTA.
// transport slots per cell whose slot codes are staged in shared memory; the
// slots' face corrections are staged in the contravariant-flux buffer once the
// divergence has consumed it (when they fit; otherwise read from global)
constexpr int SST_STAGE_SLOTS = 12;

template <int S, int NP>
__global__ void __launch_bounds__(128) k_sst_update(Geom g, Ops ops, Faces fc, SstArgs a, int cell_base,
                                                    int cell_end) {
  constexpr int CPB = SstTile<S>::CPB;
  // point values packed by k_sst_point, row stride 9: rho (clamped as the
  // reference's), u, v, w, k, omega, gamma_k, gamma_w
  __shared__ double sP[CPB * S * 9];
  __shared__ double gc[CPB * S * 3 * 2];  // reference-space grads of k, w
  // contravariant fluxes (conv k, diff k, conv w, diff w); then the face
  // corrections of the tile's transport slots (slot j's face rows at Ft + j*NP*4)
  __shared__ __align__(16) double Ft[CPB * S * 3 * 4];
  // inverse Jacobians (rows of 9) until the fluxes are formed; then R (volume
  // residuals, then with the interface corrections), T (transport k, w +
  // padding for the outlier helper) and Ref
  __shared__ double X[CPB * S * 14];
  __shared__ double sRd[CPB * S];         // det, then 1 / det
  __shared__ double work[CPB * OUT_WORK];
  __shared__ double sG[8];                // g_left, g_right
  __shared__ int sCode[CPB * SST_STAGE_SLOTS];
  __shared__ int sDfp[3 * S], sDco[3 * S];
  double* sInv = X;
  double* R = X;
  double* T = X + CPB * S * 4;
  double* Ref = X + CPB * S * 9;
  const int e0 = cell_base + blockIdx.x * CPB;
  const int nc = min(CPB, cell_end - e0);
  const int ct = cell_type(g, e0);
  // the tile's transport slots are contiguous (cell-major)
  const int k_beg = fc.tslot_ptr[e0], k_end = fc.tslot_ptr[e0 + nc];
  const bool staged = (k_end - k_beg) * NP * 4 <= CPB * S * 12 && k_end - k_beg <= CPB * SST_STAGE_SLOTS;
  double* sC = Ft;
  // the tile's blocks are contiguous: asynchronous copies, all in flight at once
  {
    const double* pb = a.sp8 + (size_t)e0 * S * 8;
    for (int t = threadIdx.x; t < nc * S * 8; t += blockDim.x) cp_async8(sP + (t >> 3) * 9 + (t & 7), pb + t);
    const double* ib = g.inv + (size_t)e0 * S * 9;
    for (int t = threadIdx.x; t < nc * S * 9; t += blockDim.x) cp_async8(sInv + t, ib + t);
    for (int t = threadIdx.x; t < nc * S; t += blockDim.x) cp_async8(sRd + t, g.det + (size_t)e0 * S + t);
    if (staged)
      for (int t = threadIdx.x; t < k_end - k_beg; t += blockDim.x) sCode[t] = __ldg(fc.tslot + k_beg + t);
    for (int t = threadIdx.x; t < 3 * S; t += blockDim.x) {
      sDfp[t] = __ldg(ops.dist_fp + t);
      sDco[t] = __ldg(ops.dist_co + t);
    }
    if (threadIdx.x < 4) {
      constexpr int N1D = S == 1 ? 1 : (S == 8 ? 2 : (S == 27 ? 3 : 4));
      sG[threadIdx.x] = threadIdx.x < N1D ? ops.g_left[threadIdx.x] : 0.0;
      sG[4 + threadIdx.x] = threadIdx.x < N1D ? ops.g_right[threadIdx.x] : 0.0;
    }
    cp_async_wait_all();
  }
  __syncthreads();
  const double* fl = sP + 4;  // k, w, gamma_k, gamma_w of point p at fl[p * 9 + 0..3]
  // grad k, grad w in reference space (D3g rows s*3+m) as one FP64
  // tensor-core product: columns (cell, field)
  {
    dmma_product_f(
        3 * S, 2 * nc, S, ops.fD3g[ct],
        [&](int j, int col) { return fl[((col >> 1) * S + j) * 9 + (col & 1)]; },
        [&](int r, int col, double x) { gc[((col >> 1) * S * 3 + r) * 2 + (col & 1)] = x; });
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nc * S; t += blockDim.x) {
    const double* inv = sInv + t * 9;
    // adjugate rows det * inv, formed here exactly as at create
    const double det = sRd[t];
    double adj[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) adj[k] = det * inv[k];
    const double* pv = sP + t * 9;  // rho = max(U0, 1e-10) and u = U1..3 / rho, as formed by k_sst_point
    const double rho = pv[0];
    const double vel[3] = {pv[1], pv[2], pv[3]};
    for (int q = 0; q < 2; ++q) {
      double gphys[3];
      for (int n = 0; n < 3; ++n) {
        double acc = 0.0;
        for (int m = 0; m < 3; ++m) acc += gc[(t * 3 + m) * 2 + q] * inv[m * 3 + n];
        gphys[n] = acc;
      }
      const double phi = fl[t * 9 + q];
      const double gam = fl[t * 9 + 2 + q];
      double Fc[3], Fd[3];
      for (int d = 0; d < 3; ++d) {
        Fc[d] = (rho * vel[d]) * phi;
        Fd[d] = gam * gphys[d];
      }
      for (int m = 0; m < 3; ++m) {
        Ft[(t * 3 + m) * 4 + 2 * q] = adj[m * 3 + 0] * Fc[0] + adj[m * 3 + 1] * Fc[1] + adj[m * 3 + 2] * Fc[2];
        Ft[(t * 3 + m) * 4 + 2 * q + 1] = adj[m * 3 + 0] * Fd[0] + adj[m * 3 + 1] * Fd[1] + adj[m * 3 + 2] * Fd[2];
      }
    }
  }
  __syncthreads();
  // one reciprocal of det per point: each use differs from a division by det
  // by at most an ulp
  for (int t = threadIdx.x; t < nc * S; t += blockDim.x) sRd[t] = 1.0 / sRd[t];
  __syncthreads();
  // divergence sum_{j,m} D[s,j,m] Ft[j,m] as one FP64 tensor-core product
  // (K = (j, m), columns (cell, field)); then the face corrections of every
  // face side in ascending color order
  {
    dmma_product_f(
        S, 4 * nc, 3 * S, ops.fD3[ct],
        [&](int k, int col) { return Ft[((col >> 2) * S * 3 + k) * 4 + (col & 3)]; },
        [&](int s, int col, double x) {
          const int b = col >> 2;
          R[(b * S + s) * 4 + (col & 3)] = -x * sRd[b * S + s];
        });
  }
  // the fluxes are consumed: the slots' face corrections arrive in their space
  __syncthreads();
  if (staged) {
    for (int t = threadIdx.x; t < (k_end - k_beg) * NP * 2; t += blockDim.x) {
      const int j = t / (NP * 2), q = t - j * (NP * 2);
      const int face = sCode[j] >> 4;
      cp_async16(sC + j * NP * 4 + 2 * q, a.cfp + (size_t)face * NP * 4 + 2 * q);
    }
    cp_async_wait_all();
  }
  __syncthreads();
  // one thread per point, all four fields, slots in order
  for (int p = threadIdx.x; p < nc * S; p += blockDim.x) {
    const int s = p % S;
    const int e = e0 + p / S;
    const double rdj = sRd[p];
    double C[4] = {0.0, 0.0, 0.0, 0.0};
    const int sb = fc.tslot_ptr[e], se = fc.tslot_ptr[e + 1];
    for (int k = sb; k < se; ++k) {
      const int code = staged ? sCode[k - k_beg] : __ldg(fc.tslot + k);
      const int ax = (code >> 2) & 3;
      const double gw = sG[((code & 1) ? 4 : 0) + sDco[ax * S + s]];
      const int fp = sDfp[ax * S + s];
      double2 c01, c23;
      if (staged) {
        const double2* cr = reinterpret_cast<const double2*>(sC + ((k - k_beg) * NP + fp) * 4);
        c01 = cr[0];
        c23 = cr[1];
      } else {
        const double2* cr = reinterpret_cast<const double2*>(a.cfp + ((size_t)(code >> 4) * NP + fp) * 4);
        c01 = __ldg(cr);
        c23 = __ldg(cr + 1);
      }
      const double cv[4] = {c01.x, c01.y, c23.x, c23.y};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double contrib = gw * cv[q];
        if (code & 2) C[q] += contrib * rdj;
        else C[q] -= contrib * rdj;
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) Ref[p * 4 + q] = C[q];  // staged: R is complete only after the barrier below
  }
  __syncthreads();
  // the fluxes are consumed: their space receives the tile's point sources
  // (Sk, Sw, beta, ...) and dt by asynchronous copies for the final update
  double* sPt = Ft;
  double* sDtS = Ft + CPB * S * 5;
  {
    const double* pb = a.pt + (size_t)e0 * S * 5;
    for (int t = threadIdx.x; t < nc * S * 5; t += blockDim.x) cp_async8(sPt + t, pb + t);
    for (int t = threadIdx.x; t < nc * S; t += blockDim.x) cp_async8(sDtS + t, a.dt + (size_t)e0 * S + t);
    cp_async_commit();
  }
  for (int p = threadIdx.x; p < nc * S; p += blockDim.x) {
    const double rho = sP[p * 9];
    const double* Cp = Ref + p * 4;
    const double conv_k = R[p * 4 + 0] + Cp[0];
    const double diff_k = R[p * 4 + 1] - Cp[1];
    const double conv_w = R[p * 4 + 2] + Cp[2];
    const double diff_w = R[p * 4 + 3] - Cp[3];
    T[p * 5 + 0] = (conv_k + diff_k) / fmax(rho, 1e-10);
    T[p * 5 + 1] = (conv_w + diff_w) / fmax(rho, 1e-10);
    T[p * 5 + 2] = 0.0; T[p * 5 + 3] = 0.0; T[p * 5 + 4] = 0.0;
  }
  __syncthreads();
  for (int p = threadIdx.x; p < nc * S; p += blockDim.x) {
    Ref[p * 5 + 0] = fl[p * 9 + 0];
    Ref[p * 5 + 1] = fl[p * 9 + 1];
    Ref[p * 5 + 2] = 0.0; Ref[p * 5 + 3] = 0.0; Ref[p * 5 + 4] = 0.0;
  }
  __syncthreads();
  cp_async_wait0();  // published by the barriers inside the outlier pass
  suppress_outliers_blocks<S>(T, Ref, 5, nc, work);
  for (int t = threadIdx.x; t < nc * S; t += blockDim.x) {
    const size_t p = (size_t)e0 * S + t;
    const double rho = sP[t * 9];
    const double tk = dfinite(T[t * 5 + 0]);
    const double tw = dfinite(T[t * 5 + 1]);
    const double* pt = sPt + t * 5;
    const double dts = sDtS[t];
    const double kf = fl[t * 9 + 0], wf = fl[t * 9 + 1];
    const double wo = fmax(wf, 1e-10);
    const double dkd = dfinite((pt[0] / fmax(rho, 1e-10)) / (1.0 + dts * (SST_BSTAR * wo)));
    const double dwd = dfinite((pt[1] / fmax(rho, 1e-10)) / (1.0 + dts * (pt[2] * wo)));
    const double kt = dfinite(dkd + tk);
    const double wt = dfinite(dwd + tw);
    double kn = kf + dts * kt;
    double wn = wf + dts * wt;
    if (!isfinite(kn)) kn = 1e-12;
    if (!isfinite(wn)) wn = 1e-12;
    a.k[p] = fmax(kn, 1e-12);
    a.w[p] = fmax(wn, 1e-12);
    if (a.dbg) {
      a.dbg[p * 4 + 0] = pt[0];
      a.dbg[p * 4 + 1] = pt[1];
      a.dbg[p * 4 + 2] = tk;
      a.dbg[p * 4 + 3] = tw;
    }
  }
}

// local time step per solution point (core/fr_solver/cfl.py:12-147)
__global__ void k_local_dt(Geom g, int S, int order, const double* __restrict__ U, int nv,
                           const double* __restrict__ nut, double mu, double* __restrict__ dt) {
  const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= (size_t)g.N * S) return;
  const int e = (int)(p / S);
  const double* u = U + p * nv;
  const double rho = fmax(u[0], 1e-10);
  const double ux = u[1] / rho, uy = u[2] / rho, uz = u[3] / rho;
  const double ke = 0.5 * (ux * ux + uy * uy + uz * uz);
  const double pr = fmax((u[4] - rho * ke) * 0.4, 1.0);
  const double a = sqrt(fmax(1.4 * pr / fmax(rho, 1e-10), 1e-10));
  const double vm = sqrt(ux * ux + uy * uy + uz * uz);
  const double wave = fmax(vm + a, 1e-10);
  const double h = g.hvol[e];  // pow(|volume|, 1/3), formed at create
  const double CFL = 0.1;
  const double fa = 1.0 / (2 * order + 1);
  const double fv = 1.0 / ((2 * order + 1) * (2 * order + 1));
  const double dt_adv = CFL * fa * h / wave;
  const double mu_eff = nut ? mu + rho * nut[p] : mu;
  const double dt_visc = 0.25 * CFL * fv * rho * (h * h) / fmax(mu_eff, 1e-30);
  const double dt_geo = CFL * fabs(g.det[p]) / fmax(g.mfs[p] * wave, 1e-300);
  dt[p] = fmin(fmin(dt_adv, dt_visc), dt_geo);
}

}  // namespace afr
