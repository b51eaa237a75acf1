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
  const double* PF;     // (N,S,18) point fields of Ucur (k_pre)
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
// per-point pre-pass: PF (N,S,18) = primitive q(5) (no pressure floor,
// core/fr_residual/inviscid.py:38-47), grads of u,v,w (9) and T (3)
// (core/fr_operators/gradients.py:23-64 as used by
// core/fr_residual/viscous_flux.py:161-166), mu_t = max(rho,1e-10) * nu_t (1)
// ---------------------------------------------------------------------------
constexpr int PFW = 18;

template <int S>
__global__ void __launch_bounds__(128) k_pre(Geom g, Ops ops, const double* __restrict__ U, int nv,
                                             const double* __restrict__ nut, int want_grads,
                                             double* __restrict__ PF) {
  __shared__ double f[S * 4];
  __shared__ double gc[S * 3 * 4];
  const int e = blockIdx.x;
  const int ct = cell_type(g, e);
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    double q[5];
    const double* u = U + ((size_t)e * S + s) * nv;
    cons_to_prim(u, q);
    double* o = PF + ((size_t)e * S + s) * PFW;
    for (int v = 0; v < 5; ++v) o[v] = q[v];
    o[17] = nut ? fmax(u[0], 1e-10) * nut[(size_t)e * S + s] : 0.0;
    f[s * 4 + 0] = q[1];
    f[s * 4 + 1] = q[2];
    f[s * 4 + 2] = q[3];
    f[s * 4 + 3] = q[4] / (fmax(q[0], 1e-10) * R_AIR);
  }
  if (!want_grads) return;
  __syncthreads();
  block_gemm<S * 3, 4, S>(gc, 4, ops.D3g[ct], S, f, 4);
  __syncthreads();
  for (int t = threadIdx.x; t < S * 12; t += blockDim.x) {
    const int s = t / 12, c = t % 12;
    const int q = c / 3, n = c % 3;  // c = q*3+n: q in (u,v,w,T)
    const double* inv = g.inv + ((size_t)e * S + s) * 9;
    double acc = 0.0;
    for (int m = 0; m < 3; ++m) acc += gc[(s * 3 + m) * 4 + q] * inv[m * 3 + n];
    PF[((size_t)e * S + s) * PFW + 5 + c] = acc;
  }
}

// ---------------------------------------------------------------------------
// fused stage kernel, one cell per CTA: volume terms, every face slot of the
// cell (own-side extrapolation, neighbour-side gather, AUSM+up / BR1 fluxes),
// correction lifting in ascending color order, outlier suppression, then
// (stage >= 0) the SSP-RK3 Shu-Osher combination, positivity projection and
// modal filter (core/time_integration/base.py:250-335,
// core/time_integration/positivity.py:13-45, core/fr_solver/filter.py:29-42).
// The inviscid volume divergence uses W = f2c * D_fine folded at create time.
// ---------------------------------------------------------------------------
constexpr int NSLOT = 5;   // a prism has 5 cube faces, a tet 4: one primary slot each
constexpr int NSRC = 2 * NSLOT;
constexpr int STAGE_THREADS = 256;

// interpolation sources staged in shared memory per cell (the rest is read
// from global memory): all of them at P1/P2, four at P3
template <int S>
struct Staging {
  static constexpr int src = S >= 64 ? 4 : NSRC;
};

template <int S, int FN, int NP>
struct StageSmem {
  static constexpr int oPF = 0;                   // S*18 own point fields
  static constexpr int oAdj = oPF + S * PFW;      // S*9
  static constexpr int oU = oAdj + S * 9;         // S*8 own state rows
  static constexpr int oDet = oU + S * 8;         // S
  static constexpr int oRi = oDet + S;            // S*5
  static constexpr int oRv = oRi + S * 5;         // S*5
  static constexpr int oJ = oRv + S * 5;          // NSLOT*NP*10 face jumps
  static constexpr int oBig = oJ + NSLOT * NP * 10;
  // slot phase: own extrapolation (21) and neighbour gather (18) per flux point
  static constexpr int sOwn = 0;
  static constexpr int sOth = sOwn + NSLOT * NP * 21;
  static constexpr int sEnd = sOth + NSLOT * NP * 18;
  // volume phase (aliases the slot scratch)
  static constexpr int vQf = 0;                   // FN*5
  static constexpr int vFt = vQf + FN * 5;        // FN*15
  static constexpr int vGt = vFt + FN * 15;       // S*15
  static constexpr int vEnd = vGt + S * 15;
  static constexpr int big = sEnd > vEnd ? sEnd : vEnd;
  static constexpr int work = oBig + big;         // 24 doubles for reductions
  static constexpr int oSM = work + 24;           // staged source matrices
  static constexpr int oSC = oSM + Staging<S>::src * NP * S;  // staged neighbour point fields
  static constexpr int total = oSC + Staging<S>::src * S * PFW;
};

template <int S, int FN, int NP>
__global__ void __launch_bounds__(STAGE_THREADS, 2) k_stage(Geom g, Ops ops, Faces fc, Bc bc, StageArgs a) {
  using L = StageSmem<S, FN, NP>;
  extern __shared__ double sm[];
  double* sPF = sm + L::oPF;
  double* sAdj = sm + L::oAdj;
  double* sU = sm + L::oU;
  double* sDet = sm + L::oDet;
  double* sRi = sm + L::oRi;
  double* sRv = sm + L::oRv;
  double* sJ = sm + L::oJ;
  double* big = sm + L::oBig;
  double* work = sm + L::work;
  __shared__ int slF[NSLOT], slAx[NSLOT], slOwn[NSLOT], slBnd[NSLOT];
  __shared__ double slSide[NSLOT];
  __shared__ const double* slE[NSLOT];
  __shared__ int slSrc[NSLOT + 1];                 // sources of slot sl: [slSrc[sl], slSrc[sl+1])
  __shared__ const double* srcM[NSRC];             // source matrix (global)
  __shared__ int srcCell[NSRC], srcStage[NSRC];    // neighbour cell, staged cell slot or -1
  __shared__ int n_src, n_ucell;
  __shared__ int ucell[NSRC];
  constexpr int MAXST = Staging<S>::src;
  double* sMs = sm + L::oSM;
  double* sNs = sm + L::oSC;

  const int e = blockIdx.x;
  const int ct = cell_type(g, e);
  const int nv = a.nv;
  const bool visc = !a.inviscid_only;
  const int tid = threadIdx.x;
  const int s_beg = fc.slot_ptr[e];
  const int nsl = min(fc.slot_ptr[e + 1] - s_beg, NSLOT);

  // ---- phase 0: own cell, slot metadata, staged sources ----
  {
    const double* pf = a.PF + (size_t)e * S * PFW;
    for (int t = tid; t < S * PFW; t += blockDim.x) sPF[t] = pf[t];
    const double* ad = g.adj + (size_t)e * S * 9;
    for (int t = tid; t < S * 9; t += blockDim.x) sAdj[t] = ad[t];
    const double* u = a.Ucur + (size_t)e * S * nv;
    for (int t = tid; t < S * nv; t += blockDim.x) sU[(t / nv) * 8 + t % nv] = u[t];
    for (int t = tid; t < S; t += blockDim.x) sDet[t] = g.det[(size_t)e * S + t];
    if (tid == 0) {
      if (fc.slot_ptr[e + 1] - s_beg > NSLOT) atomicOr(a.status, DS_BAD_INDEX);
      int k = 0, nu = 0;
      for (int sl = 0; sl < nsl; ++sl) {
        const int code = fc.slot[s_beg + sl];
        const int f = code >> 1;
        const bool own = (code & 1) == 0;
        const int ax = own ? fc.o_axis[f] : fc.n_axis[f];
        const double side = own ? fc.o_side[f] : fc.n_side[f];
        slF[sl] = f;
        slOwn[sl] = own;
        slAx[sl] = ax;
        slSide[sl] = side;
        slBnd[sl] = fc.is_bnd[f];
        slE[sl] = ops.extrap + (((size_t)ct * 3 + ax) * 2 + (side < 0.0 ? 0 : 1)) * NP * S;
        slSrc[sl] = k;
        if (slBnd[sl]) continue;
        const int c0 = own ? fc.nb_c0[f] : fc.ow_c0[f];
        const int i1 = own ? fc.nb_i1[f] : fc.ow_i1[f];
        for (int src = 0; src < 2; ++src) {
          const int c = src == 0 ? c0 : (i1 >= 0 ? (own ? fc.nb_c1[i1] : fc.ow_c1[i1]) : -1);
          if (c < 0) continue;
          srcM[k] = src == 0 ? (own ? fc.nb_m0 : fc.ow_m0) + (size_t)f * NP * S
                             : (own ? fc.nb_m1 : fc.ow_m1) + (size_t)i1 * NP * S;
          srcCell[k] = c;
          int st = -1;
          for (int j = 0; j < nu; ++j)
            if (ucell[j] == c) st = j;
          if (st < 0 && nu < MAXST) {
            ucell[nu] = c;
            st = nu++;
          }
          srcStage[k] = st;
          ++k;
        }
      }
      slSrc[nsl] = k;
      n_src = k;
      n_ucell = nu;
    }
  }
  __syncthreads();
  {
    const int nm = min(n_src, MAXST);
    for (int t = tid; t < nm * NP * S; t += blockDim.x) {
      const int k = t / (NP * S), r = t % (NP * S);
      sMs[t] = __ldg(srcM[k] + r);
    }
    for (int t = tid; t < n_ucell * S * PFW; t += blockDim.x) {
      const int j = t / (S * PFW), r = t % (S * PFW);
      sNs[t] = __ldg(a.PF + (size_t)ucell[j] * S * PFW + r);
    }
  }
  __syncthreads();

  // ---- phase 1: own extrapolations and neighbour gathers of every slot ----
  double* own = big + L::sOwn;  // [sl][i][21]: q(5) adj row(3) grads+mu_t(13)
  double* oth = big + L::sOth;  // [sl][i][18]: q(5) grads+mu_t(13)
  {
    const int nown3 = visc ? 7 : 3;
    const int noth3 = visc ? 6 : 2;
    const int n_own = nsl * NP * nown3;
    const int n_all = n_own + nsl * NP * noth3;
    for (int t = tid; t < n_all; t += blockDim.x) {
      if (t < n_own) {
        const int sl = t / (NP * nown3), r = t % (NP * nown3), i = r / nown3, c0 = (r % nown3) * 3;
        const double* Er = slE[sl] + i * S;
        const int ax = slAx[sl];
        double acc[3] = {0.0, 0.0, 0.0};
        for (int s = 0; s < S; ++s) {
          const double w = __ldg(Er + s);
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const int c = c0 + j;
            const double x = c < 5 ? sPF[s * PFW + c] : (c < 8 ? sAdj[s * 9 + ax * 3 + c - 5] : sPF[s * PFW + c - 3]);
            acc[j] += w * x;
          }
        }
        double* o = own + (sl * NP + i) * 21 + c0;
        for (int j = 0; j < 3; ++j) o[j] = acc[j];
      } else {
        const int u = t - n_own;
        const int sl = u / (NP * noth3), r = u % (NP * noth3), i = r / noth3, k0 = (r % noth3) * 3;
        if (slBnd[sl]) continue;
        double acc[3] = {0.0, 0.0, 0.0};
        for (int k = slSrc[sl]; k < slSrc[sl + 1]; ++k) {
          const double* Mr = (k < MAXST ? sMs + k * NP * S : srcM[k]) + i * S;
          const int st = srcStage[k];
          const double* pf = (st >= 0 ? sNs + st * S * PFW : a.PF + (size_t)srcCell[k] * S * PFW) + k0;
          for (int s = 0; s < S; ++s) {
            const double w = Mr[s];
            // the reference skips zero weights (inviscid_kernel_colored.py:117-121)
#pragma unroll
            for (int j = 0; j < 3; ++j) acc[j] += (w != 0.0) ? w * pf[s * PFW + j] : 0.0;
          }
        }
        double* o = oth + (sl * NP + i) * 18 + k0;
        for (int j = 0; j < 3; ++j) o[j] = acc[j];
      }
    }
  }
  __syncthreads();

  // ---- phase 2: pointwise interface fluxes at every (slot, flux point) ----
  double vol_o = 0.0;
  if (visc) {
    for (int s = 0; s < S; ++s) vol_o += sDet[s];
    vol_o /= S;
  }
  for (int t = tid; t < nsl * NP; t += blockDim.x) {
    const int sl = t / NP, i = t % NP;
    const double* ow = own + (sl * NP + i) * 21;
    double* ot = oth + (sl * NP + i) * 18;
    const int f = slF[sl];
    const double side = slSide[sl];
    const bool is_owner = slOwn[sl] != 0;
    const double* tn = fc.tnormal + ((size_t)f * NP + i) * 3;
    if (slBnd[sl]) {
      double qo[5], n[3], gq[5];
      for (int v = 0; v < 5; ++v) qo[v] = ow[v];
      for (int d = 0; d < 3; ++d) n[d] = tn[d];
      ghost_state(bc, fc.bc_group[f], qo, n, gq);
      for (int v = 0; v < 5; ++v) ot[v] = gq[v];
      for (int k = 0; k < 13; ++k) ot[5 + k] = ow[8 + k];
    }
    const double a0 = ow[5], a1 = ow[6], a2 = ow[7];
    double mag = sqrt(a0 * a0 + a1 * a1 + a2 * a2);
    if (mag < 1e-300) mag = 1e-300;
    double dir[3] = {a0 / mag * side, a1 / mag * side, a2 / mag * side};
    const double sg = is_owner ? 1.0 : -1.0;
    const double t0 = sg * tn[0], t1 = sg * tn[1], t2 = sg * tn[2];
    if (dir[0] * t0 + dir[1] * t1 + dir[2] * t2 < 0.5) { dir[0] = t0; dir[1] = t1; dir[2] = t2; }
    double qo[5], qn[5], Fc[5], Fp[3][5];
    for (int v = 0; v < 5; ++v) { qo[v] = ow[v]; qn[v] = ot[v]; }
    ausm_up(qo, qn, dir, Fc);
    euler_flux(qo, Fp);
    double* J = sJ + (sl * NP + i) * 10;
    for (int v = 0; v < 5; ++v) J[v] = Fc[v] * mag * side - (a0 * Fp[0][v] + a1 * Fp[1][v] + a2 * Fp[2][v]);
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
      if (slBnd[sl]) {
        // interior-penalty term on boundary faces (core/fr_operators/flux_kernels.py:140-200)
        double h = pow(vol_o, 1.0 / 3.0);
        if (h < 1e-300) h = 1e-300;
        const double eta = C_IP * (a.mu + ow[20]) / h;
        const double scale = eta * sqrt(a0 * a0 + a1 * a1 + a2 * a2) * side;
        for (int v = 1; v < 4; ++v) jv[v] += -scale * (qo[v] - qn[v]);
      }
      for (int v = 0; v < 5; ++v) J[5 + v] = jv[v];
    }
  }
  __syncthreads();

  // ---- phase 3: volume terms ----
  {
    double* Qf = big + L::vQf;
    double* Ft = big + L::vFt;
    double* Gt = big + L::vGt;
    // Q at fine points (c2f), own Q is sPF[s*18 + 0..4]
    for (int t = tid; t < FN * 5; t += blockDim.x) {
      const int i = t / 5, v = t % 5;
      const double* c = ops.c2f[ct] + i * S;
      double acc = 0.0;
      for (int s = 0; s < S; ++s) acc += __ldg(c + s) * sPF[s * PFW + v];
      Qf[t] = acc;
    }
    if (visc) {
      for (int s = tid; s < S; s += blockDim.x) {
        double q[5], G[3][5];
        const double* p = sPF + s * PFW;
        for (int v = 0; v < 5; ++v) q[v] = p[v];
        viscous_flux(q, p + 5, p + 14, a.mu, p[17], G);
        const double* am = sAdj + s * 9;
        for (int m = 0; m < 3; ++m)
          for (int v = 0; v < 5; ++v)
            Gt[(s * 3 + m) * 5 + v] = am[m * 3 + 0] * G[0][v] + am[m * 3 + 1] * G[1][v] + am[m * 3 + 2] * G[2][v];
      }
    }
    __syncthreads();
    for (int i = tid; i < FN; i += blockDim.x) {
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
    // inviscid divergence W (S x 3FN) and viscous divergence D3 (S x 3S)
    const int n_i = S * 5, n_all = visc ? 2 * S * 5 : S * 5;
    for (int t = tid; t < n_all; t += blockDim.x) {
      if (t < n_i) {
        const int s = t / 5, v = t % 5;
        const double* w = ops.W[ct] + (size_t)s * FN * 3;
        double acc = 0.0;
#pragma unroll 4
        for (int k = 0; k < FN * 3; ++k) acc += __ldg(w + k) * Ft[k * 5 + v];
        sRi[t] = -acc / sDet[s];
      } else {
        const int u = t - n_i, s = u / 5, v = u % 5;
        const double* d = ops.D3[ct] + (size_t)s * S * 3;
        double acc = 0.0;
#pragma unroll 4
        for (int k = 0; k < S * 3; ++k) acc += __ldg(d + k) * Gt[k * 5 + v];
        sRv[u] = acc / sDet[s];
      }
    }
  }
  __syncthreads();

  // ---- phase 4: lift corrections, slots in ascending color order ----
  for (int t = tid; t < S * 5; t += blockDim.x) {
    const int s = t / 5, v = t % 5;
    double ci = 0.0, cv = 0.0;
    for (int sl = 0; sl < nsl; ++sl) {
      const int ax = slAx[sl];
      const int fp = ops.dist_fp[ax * S + s];
      const double gw = (slSide[sl] < 0.0 ? ops.g_left : ops.g_right)[ops.dist_co[ax * S + s]];
      const double* J = sJ + (sl * NP + fp) * 10;
      ci += -(gw * J[v]) / sDet[s];
      if (visc) cv += (gw * J[5 + v]) / sDet[s];
    }
    sRi[t] = sRi[t] + ci;
    if (visc) sRv[t] = sRv[t] + cv;
  }
  __syncthreads();
  suppress_outliers<S>(sRi, sU, 8, work);
  if (visc) suppress_outliers<S>(sRv, sU, 8, work);

  if (a.stage < 0) {
    for (int t = tid; t < S * nv; t += blockDim.x) {
      const int s = t / nv, v = t % nv;
      if (a.Rinv) a.Rinv[(size_t)e * S * nv + t] = v < 5 ? sRi[s * 5 + v] : 0.0;
      if (a.Rvisc) a.Rvisc[(size_t)e * S * nv + t] = (v < 5 && visc) ? sRv[s * 5 + v] : 0.0;
    }
    return;
  }

  // ---- phase 5: RK stage combination + positivity (per point) ----
  double* Up = big;  // (S, 8)
  double part = 0.0;
  for (int s = tid; s < S; s += blockDim.x) {
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
  for (int t = tid; t < S * nv; t += blockDim.x) {
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
    if ((tid & 31) == 0) work[tid >> 5] = part;
    __syncthreads();
    if (tid == 0) {
      double acc = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) acc += work[w];
      a.norm_part[e] = acc;
    }
  }
}

}  // namespace afr
