// Order-0 (finite-volume) residual and update: one solution point per cell.
// Restates (paths relative to the reference's src/autoflowcfd):
//   compute_inviscid_residual_fv_p0  core/fr_residual/inviscid_p0.py:18-85 with
//                                    its kernel core/fr_residual/inviscid_p0_kernel.py:25-108
//   _precompute_ghost_states         core/fr_residual/inviscid_p0.py:112-143
//   viscous residual                 core/fr_residual/viscous_flux.py:113-302 at one point per
//                                    cell: the local gradients vanish (the derivative operator
//                                    is zero), so of the colored interface kernel
//                                    (core/fr_residual/viscous_flux_kernel.py:292-520) only the
//                                    interior-penalty term of boundary faces remains
//                                    (core/fr_operators/flux_kernels.py:140-200)
//
// Inviscid: every face record contributes AUSM+up(owner, other side) along its
// unit normal times its area, taken out of the owner and added to the
// neighbour, each divided by that cell's volume; no primary-side filtering.
// The reference keeps ONE ghost state per owner cell, overwritten face by face
// in record order, so every boundary face of a cell uses the ghost state of
// the cell's last boundary face (its normal, its boundary group).  That table
// (gface) is formed at create.  Per cell the contributions are summed in
// ascending face-record order, the order of the reference's sequential loop.
#pragma once
#include "afr_implicit.cuh"

namespace afr {

struct P0Tab {
  const int32_t* cptr;   // (N+1) per-cell face references
  const int32_t* cref;   // face << 1 | (this cell is the face's neighbour), ascending face record
  const int32_t* gface;  // (F) boundary face whose normal and group make the ghost state, -1 inside
  const int32_t* pen;    // (F) 0, or 1 | owner axis << 1 | (owner side > 0) << 3 for an owner-primary boundary face
  const double* area;    // (F) face area (true_area_weight of the single face point)
  const double* volume;  // (N) finite-volume divisor (the mesh's cell volumes at its load order)
  double* flux;          // (F, 8) AUSM+up flux * area (5), viscous penalty jump of the momentum (3)
};

// one thread per face record
__global__ void __launch_bounds__(128) k_p0_face(Geom g, Faces fc, Bc bc, P0Tab t, const double* __restrict__ U,
                                                 int nv, const double* __restrict__ nut, double mu, int visc) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= fc.F) return;
  const int o = fc.owner[f];
  const bool bnd = fc.is_bnd[f] != 0;
  double qo[5], qn[5], n[3];
  cons_to_prim(U + (size_t)o * nv, qo);
  for (int d = 0; d < 3; ++d) n[d] = fc.tnormal[(size_t)f * 3 + d];
  if (bnd) {
    const int gf = t.gface[f];
    double gn[3];
    for (int d = 0; d < 3; ++d) gn[d] = fc.tnormal[(size_t)gf * 3 + d];
    ghost_state(bc, fc.bc_group[gf], qo, gn, qn);
  } else {
    cons_to_prim(U + (size_t)fc.neighbor[f] * nv, qn);
  }
  double Fc[5];
  ausm_up(qo, qn, n, Fc);
  const double A = t.area[f];
  double* out = t.flux + (size_t)f * 8;
  for (int v = 0; v < 5; ++v) out[v] = Fc[v] * A;
  double jv[3] = {0.0, 0.0, 0.0};
  const int pc = t.pen[f];
  if (visc && pc) {
    // the viscous path's own ghost state of this face
    double gq[5];
    ghost_state(bc, fc.bc_group[f], qo, n, gq);
    const int ax = (pc >> 1) & 3;
    const double side = (pc & 8) ? 1.0 : -1.0;
    const double* ad = g.adj + (size_t)o * 9 + ax * 3;
    const double a0 = ad[0], a1 = ad[1], a2 = ad[2];
    double h = pow(g.det[o], 1.0 / 3.0);  // cell volume scale: the mean of det over the one point
    if (h < 1e-300) h = 1e-300;
    const double mut = nut ? fmax(U[(size_t)o * nv], 1e-10) * nut[o] : 0.0;
    const double eta = C_IP * (mu + mut) / h;
    const double scale = eta * sqrt(a0 * a0 + a1 * a1 + a2 * a2) * side;
    for (int v = 1; v < 4; ++v) jv[v - 1] = -scale * (qo[v] - gq[v]);
  }
  for (int v = 0; v < 3; ++v) out[5 + v] = jv[v];
}

// one thread per cell: gather the face contributions, then (stage >= 0) the
// SSP-RK3 combination, positivity and the (1 x 1) modal filter.  Outlier
// suppression is the identity for one point per cell (a value never exceeds
// 1e4 times itself), so it is not run.
__global__ void __launch_bounds__(128) k_p0_cell(Geom g, Ops ops, Faces fc, P0Tab t, StageArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.N) return;
  const int nv = a.nv;
  const bool visc = !a.inviscid_only;
  double ri[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  const double rvol = 1.0 / t.volume[c];
  for (int k = t.cptr[c]; k < t.cptr[c + 1]; ++k) {
    const int code = t.cref[k];
    const double* F = t.flux + (size_t)(code >> 1) * 8;
    if (code & 1) {
      for (int v = 0; v < 5; ++v) ri[v] += F[v] * rvol;
    } else {
      for (int v = 0; v < 5; ++v) ri[v] -= F[v] * rvol;
    }
  }
  // viscous corrections of the owner-primary boundary slots, ascending color
  double rv[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (visc) {
    const double det = g.det[c];
    for (int k = fc.slot_ptr[c]; k < fc.slot_ptr[c + 1]; ++k) {
      const int code = fc.slot[k];
      if (code & 1) continue;  // neighbour sides never carry the penalty
      const int f = code >> 1;
      const int pc = t.pen[f];
      if (!pc) continue;
      const double gw = (pc & 8) ? ops.g_right[0] : ops.g_left[0];
      const double* J = t.flux + (size_t)f * 8 + 5;
      for (int v = 1; v < 4; ++v) rv[v] += (gw * J[v - 1]) / det;
    }
  }
  const size_t p = (size_t)c;
  if (a.stage < 0) {
    for (int v = 0; v < nv; ++v) {
      if (a.Rinv) a.Rinv[p * nv + v] = v < 5 ? ri[v] : 0.0;
      if (a.Rvisc) a.Rvisc[p * nv + v] = (v < 5 && visc) ? rv[v] : 0.0;
    }
    return;
  }
  double Lr[8], un[8];
  double sq_sum = 0.0;
#pragma unroll
  for (int v = 0; v < 8; ++v) Lr[v] = v < 5 ? ri[v] + (visc ? rv[v] : 0.0) : 0.0;
#pragma unroll
  for (int v = 0; v < 8; ++v)
    if (v < nv) sq_sum += Lr[v] * Lr[v];
  const double dts = a.dt[p];
  const double* u0 = a.U0 + p * nv;
  const double* uc = a.Ucur + p * nv;
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    if (v >= nv) {
      un[v] = 0.0;
    } else if (a.stage == 0) {
      un[v] = u0[v] + dts * Lr[v];
    } else if (a.stage == 1) {
      un[v] = (0.75 * u0[v] + 0.25 * uc[v]) + (0.25 * dts) * Lr[v];
    } else {
      un[v] = (1.0 / 3.0 * u0[v] + 2.0 / 3.0 * uc[v]) + (2.0 / 3.0 * dts) * Lr[v];
    }
  }
  positivity_point(un, nv);
  const double fm = ops.filt[cell_type(g, c)][0];
#pragma unroll
  for (int v = 0; v < 8; ++v)
    if (v < nv) a.Unext[p * nv + v] = v < 5 ? 0.0 + fm * un[v] : un[v];
  if (a.stage == 0) {
    a.norm_part[c] = 0.0 + sq_sum;
    a.norm_rho_part[c] = 0.0 + Lr[0] * Lr[0];
    if (!isfinite(sq_sum) && a.status) atomicOr(a.status, (unsigned)DS_NONFINITE);
  }
}

}  // namespace afr
