// Device-side data layout and pointwise physics for the FR residual-and-update path.
//
// Every array below lives in HBM, owned by one afr_handle (see afr_api.cu).
// Cell-major layouts follow the reference's own arrays so the C-ABI can take
// them unchanged: U (N,S,nv), det (N,S), adj/inv (N,S,3,3), face tables
// (F,...).  The pointwise functions restate the reference formulas
// (paths relative to the reference's src/autoflowcfd):
//   ausm_up          core/fr_operators/kernels.py:19-155
//   euler_flux       core/fr_operators/flux_kernels.py:28-68
//   viscous_flux     core/fr_operators/flux_kernels.py:71-137
//   ghost_state      boundary/fr_ghost_state.py:26-189
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace afr {

constexpr double GAMMA = 1.4;
constexpr double R_AIR = 287.0;
constexpr double PR = 0.72;
constexpr double PR_T = 0.9;
constexpr double C_IP = 4.0;

enum BcType : int32_t { BC_WALL = 0, BC_FARFIELD = 1, BC_INLET = 2, BC_OUTLET = 3, BC_SYMMETRY = 4 };

// Status word bits written by kernels instead of trapping (host reads them).
enum DevStatus : uint32_t { DS_OK = 0u, DS_BAD_INDEX = 1u, DS_NONFINITE = 2u };

// Per-cell-type operator set (index 0 = prism, 1 = tet), all row-major doubles.
struct Ops {
  const double* D3[2];      // (S, S, 3): D3[s*3S + j*3 + m]
  const double* D3g[2];     // (3S, S):   gradient form, row s*3+m, col j
  const double* c2f[2];     // (Fn, S)
  const double* Dfine[2];   // (Fn, Fn*3)
  const double* f2c[2];     // (S, Fn)
  const double* W[2];       // (S, 3Fn) = f2c * D_fine, folded once at create
  const double* filt[2];    // (S, S)
  const double* extrap;     // (2, 3, 2, P, S)
  const double* g_left;     // (n1d)
  const double* g_right;    // (n1d)
  const int32_t* dist_fp;   // (3, S)
  const int32_t* dist_co;   // (3, S)
};

struct Geom {
  int32_t N, n_prism;
  const double* det;        // (N, S)
  const double* inv;        // (N, S, 3, 3)
  const double* adj;        // (N, S, 3, 3)  det * inv, formed once at create
  const double* adj_fine;   // (N, Fn, 3, 3)
  const double* volume;     // (N)
  const double* mfs;        // (N, S) sum_m |adj[m,:]|
  const double* wall_dist;  // (N, S) or null
};

// Face records.  A "slot" is one side of one face record whose own
// extrapolation + correction lifting runs on this cell; slots of a cell are
// stored in ascending face-color order, which is the order the reference's
// colored kernels add corrections into a cell.
struct Faces {
  int32_t F;
  const int32_t* owner;       // (F)
  const int32_t* neighbor;    // (F), -1 on boundary
  const int8_t* o_axis;       // (F)
  const int8_t* n_axis;       // (F)
  const double* o_side;       // (F) +-1
  const double* n_side;       // (F)
  const uint8_t* is_bnd;      // (F)
  const double* tnormal;      // (F, P, 3)
  const int32_t* nb_c0;       // (F) neighbor-side sources (owner side reads)
  const double* nb_m0;        // (F, P, S)
  const int32_t* nb_i1;       // (F) index into the compact second source, -1 if none
  const int32_t* nb_c1;       // (n1)
  const double* nb_m1;        // (n1, P, S)
  const int32_t* ow_c0;       // owner-side sources (neighbor side reads)
  const double* ow_m0;
  const int32_t* ow_i1;
  const int32_t* ow_c1;
  const double* ow_m1;
  const int32_t* bc_group;    // (F) row of the BC table
  // residual slots: primary sides, ascending color
  const int32_t* slot_ptr;    // (N+1)
  const int32_t* slot;        // face*2 + (0 owner, 1 neighbor)
  // transport slots: every face side (owner always, neighbor if interior)
  const int32_t* tslot_ptr;   // (N+1)
  const int32_t* tslot;
};

struct Bc {
  int32_t n;
  const int32_t* type;
  const int32_t* noslip;
  const double* wall_vel;     // (n,3)
  const double* Q;            // (n,5)
  const double* p_out;        // (n)
};

// ---------------------------------------------------------------------------
// pointwise physics
// ---------------------------------------------------------------------------
__device__ __forceinline__ void euler_flux(const double q[5], double F[3][5]) {
  const double rho = q[0], u = q[1], v = q[2], w = q[3], p = q[4];
  const double rs = fmax(rho, 1e-10);
  const double ke = 0.5 * (u * u + v * v + w * w);
  const double e_int = p / ((GAMMA - 1.0) * rs);
  const double rhoE = rho * (e_int + ke);
  const double H = (rhoE + p) / rs;
  const double mf0 = rho * u, mf1 = rho * v, mf2 = rho * w;
  F[0][0] = mf0; F[0][1] = mf0 * u + p; F[0][2] = mf0 * v;     F[0][3] = mf0 * w;     F[0][4] = rho * H * u;
  F[1][0] = mf1; F[1][1] = mf1 * u;     F[1][2] = mf1 * v + p; F[1][3] = mf1 * w;     F[1][4] = rho * H * v;
  F[2][0] = mf2; F[2][1] = mf2 * u;     F[2][2] = mf2 * v;     F[2][3] = mf2 * w + p; F[2][4] = rho * H * w;
}

__device__ __forceinline__ double sq(double x) { return x * x; }

__device__ __forceinline__ void ausm_up(const double qL[5], const double qR[5], const double n[3], double out[5]) {
  const double alpha = 0.1875, beta = 0.5, Kp = 0.25, Ku = 0.75, sigma_p = 1.0, ma_ref = 0.1;
  const double rhoL = fmax(qL[0], 1e-6), rhoR = fmax(qR[0], 1e-6);
  const double pL = fmax(qL[4], 10.0), pR = fmax(qR[4], 10.0);
  const double uL = qL[1], vL = qL[2], wL = qL[3];
  const double uR = qR[1], vR = qR[2], wR = qR[3];
  const double unL = uL * n[0] + vL * n[1] + wL * n[2];
  const double unR = uR * n[0] + vR * n[1] + wR * n[2];
  const double aL = sqrt(fmax(GAMMA * pL / rhoL, 1e-10));
  const double aR = sqrt(fmax(GAMMA * pR / rhoR, 1e-10));
  const double ML = unL / fmax(aL, 1e-10);
  const double MR = unR / fmax(aR, 1e-10);
  const double a_half = 0.5 * (aL + aR);
  const double rho_half = 0.5 * (rhoL + rhoR);
  const double Mbar2 = (sq(unL) + sq(unR)) / (2.0 * sq(a_half));
  const double M0 = fmin(1.0, fmax(Mbar2, ma_ref * ma_ref));
  double fa = sqrt(M0) * (2.0 - sqrt(M0));
  fa = fmax(fa, 1e-6);
  const double mp = (fabs(ML) >= 1.0) ? 0.5 * (ML + fabs(ML)) : 0.25 * sq(ML + 1.0) + alpha * sq(sq(ML) - 1.0);
  const double mm = (fabs(MR) >= 1.0) ? 0.5 * (MR - fabs(MR)) : -0.25 * sq(MR - 1.0) - alpha * sq(sq(MR) - 1.0);
  const double M_half = mp + mm;
  const double Mp = -(Kp / fa) * fmax(1.0 - sigma_p * Mbar2, 0.0) * (pR - pL) / (rho_half * sq(a_half));
  const double mdot = 0.5 * (rhoL * aL + rhoR * aR) * (M_half + Mp);
  const double sgnL = (ML > 0.0) ? 1.0 : ((ML < 0.0) ? -1.0 : 0.0);
  const double sgnR = (MR > 0.0) ? 1.0 : ((MR < 0.0) ? -1.0 : 0.0);
  const double PpL = (fabs(ML) >= 1.0) ? 0.5 * (1.0 + sgnL)
                                        : 0.25 * (sq(ML + 1.0) * (2.0 - ML) + beta * ML * sq(sq(ML) - 1.0));
  const double PmR = (fabs(MR) >= 1.0) ? 0.5 * (1.0 - sgnR)
                                        : 0.25 * (sq(MR - 1.0) * (2.0 + MR) - beta * MR * sq(sq(MR) - 1.0));
  const double p_half = PpL * pL + PmR * pR - Ku * PpL * PmR * (rhoL + rhoR) * fa * a_half * (unR - unL);
  const bool up = mdot >= 0.0;
  out[0] = mdot;
  out[1] = mdot * (up ? uL : uR) + p_half * n[0];
  out[2] = mdot * (up ? vL : vR) + p_half * n[1];
  out[3] = mdot * (up ? wL : wR) + p_half * n[2];
  const double hL = GAMMA / (GAMMA - 1.0) * pL / rhoL + 0.5 * (sq(uL) + sq(vL) + sq(wL));
  const double hR = GAMMA / (GAMMA - 1.0) * pR / rhoR + 0.5 * (sq(uR) + sq(vR) + sq(wR));
  out[4] = mdot * (up ? hL : hR);
}

// gv[a*3+b] = d u_a / d x_b, gT[3], viscous flux G (3,5)
__device__ __forceinline__ void viscous_flux(const double q[5], const double gv[9], const double gT[3], double mu,
                                             double mu_t, double G[3][5]) {
  const double mt = mu + mu_t;
  const double S00 = gv[0], S11 = gv[4], S22 = gv[8];
  const double S01 = 0.5 * (gv[1] + gv[3]);
  const double S02 = 0.5 * (gv[2] + gv[6]);
  const double S12 = 0.5 * (gv[5] + gv[7]);
  const double div = gv[0] + gv[4] + gv[8];
  const double lam = -2.0 / 3.0 * mt;
  const double t00 = 2.0 * mt * S00 + lam * div;
  const double t11 = 2.0 * mt * S11 + lam * div;
  const double t22 = 2.0 * mt * S22 + lam * div;
  const double t01 = 2.0 * mt * S01, t02 = 2.0 * mt * S02, t12 = 2.0 * mt * S12;
  const double cp = GAMMA * R_AIR / (GAMMA - 1.0);
  const double k = mu * cp / PR + mu_t * cp / PR_T;
  const double u = q[1], v = q[2], w = q[3];
  G[0][0] = 0.0; G[0][1] = t00; G[0][2] = t01; G[0][3] = t02;
  G[1][0] = 0.0; G[1][1] = t01; G[1][2] = t11; G[1][3] = t12;
  G[2][0] = 0.0; G[2][1] = t02; G[2][2] = t12; G[2][3] = t22;
  G[0][4] = (u * t00 + v * t01 + w * t02) + (-k * gT[0]);
  G[1][4] = (u * t01 + v * t11 + w * t12) + (-k * gT[1]);
  G[2][4] = (u * t02 + v * t12 + w * t22) + (-k * gT[2]);
}

// conserved -> primitive without pressure floor (core/fr_residual/inviscid.py:38-47)
__device__ __forceinline__ void cons_to_prim(const double* U, double q[5]) {
  const double rho = fmax(U[0], 1e-10);
  const double u = U[1] / rho, v = U[2] / rho, w = U[3] / rho;
  const double E = U[4] / rho;
  const double ke = 0.5 * (u * u + v * v + w * w);
  q[0] = rho; q[1] = u; q[2] = v; q[3] = w;
  q[4] = (GAMMA - 1.0) * rho * (E - ke);
}

// boundary ghost state at one flux point (boundary/fr_ghost_state.py:26-189)
__device__ __forceinline__ void ghost_state(const Bc& bc, int code, const double qo[5], const double n[3],
                                            double g[5]) {
  for (int v = 0; v < 5; ++v) g[v] = qo[v];
  const int t = bc.type[code];
  const double vn = qo[1] * n[0] + qo[2] * n[1] + qo[3] * n[2];
  if (t == BC_WALL) {
    if (bc.noslip[code]) {
      for (int d = 0; d < 3; ++d) g[1 + d] = 2.0 * bc.wall_vel[code * 3 + d] - qo[1 + d];
    } else {
      for (int d = 0; d < 3; ++d) g[1 + d] = qo[1 + d] - 2.0 * vn * n[d];
    }
  } else if (t == BC_FARFIELD) {
    for (int v = 0; v < 5; ++v) g[v] = bc.Q[code * 5 + v];
  } else if (t == BC_INLET) {
    if (vn < 0.0)
      for (int v = 0; v < 5; ++v) g[v] = bc.Q[code * 5 + v];
  } else if (t == BC_OUTLET) {
    if (vn > 0.0) g[4] = bc.p_out[code];
  } else if (t == BC_SYMMETRY) {
    for (int d = 0; d < 3; ++d) g[1 + d] = qo[1 + d] - 2.0 * vn * n[d];
  }
}

}  // namespace afr
