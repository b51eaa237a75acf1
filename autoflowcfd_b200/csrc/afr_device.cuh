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
enum DevStatus : uint32_t {
  DS_OK = 0u,
  DS_BAD_INDEX = 1u,
  DS_NONFINITE = 2u,
  DS_TC_TIMEOUT = 4u      // a tensor-core completion wait ran out (mixed form)
};

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
  // fragment-major images of the A operands of the FP64 tensor-core products
  // (element (m, k) of an M x K operator at [((m/8) * ceil(K/4) + k/4) * 32 +
  // (m%8) * 4 + k%4], zero outside the operator): one warp's fragment load is
  // 256 contiguous bytes
  const double* fD3[2];     // D3 as (S, 3S)
  const double* fD3g[2];    // D3g (3S, S)
  const double* fc2f[2];    // c2f (Fn, S)
  const double* fW[2];      // W (S, 3Fn)
  const double* ffilt[2];   // filt (S, S)
  const double* fextrap;    // extrap: 12 images of (P, S), ceil(P/8) * ceil(S/4) * 32 doubles each
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
  const double* hvol;       // (N) |volume|^(1/3), the local-dt length (formed once at create)
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
  // Interpolation matrices stored transposed, (rows, S, P) with the face
  // point fastest, one matrix per record through a row index: a shared table
  // of the distinct matrices when the mesh gives one (a few dozen on
  // generated meshes), else the dense per-record arrays with identity
  // indices.  fmat() gives record r's face point i; weight s is at [s * P].
  const int32_t* nb_c0;       // (F) neighbor-side sources (owner side reads)
  const double* nb_m0;        // matrices of nb_m0i
  const int32_t* nb_m0i;      // (F)
  const int32_t* nb_i1;       // (F) index into the compact second source, -1 if none
  const int32_t* nb_c1;       // (n1)
  const double* nb_m1;
  const int32_t* nb_m1i;      // (n1)
  const int32_t* ow_c0;       // owner-side sources (neighbor side reads)
  const double* ow_m0;
  const int32_t* ow_m0i;
  const int32_t* ow_i1;
  const int32_t* ow_c1;
  const double* ow_m1;
  const int32_t* ow_m1i;
  const int32_t* bc_group;    // (F) row of the BC table
  // residual slots: primary sides, ascending color
  const int32_t* slot_ptr;    // (N+1)
  const int32_t* slot;        // face*2 + (0 owner, 1 neighbor)
  // transport slots: every face side (owner always, neighbor if interior)
  const int32_t* tslot_ptr;   // (N+1)
  const int32_t* tslot;       // face << 4 | axis << 2 | (neighbor side) << 1 | (side > 0)
};

// face point i of record r in an indexed, transposed matrix array: weight s at [s * NP]
__device__ __forceinline__ const double* fmat(const double* m, const int32_t* mi, size_t r, int i, int NP, int S) {
  return m + (size_t)mi[r] * S * NP + i;
}

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
// The pointwise functions are templates on the real type T: the FP64 path
// instantiates them with double (every literal is converted with T(..), so the
// double instantiation is the plain double expression); the mixed-precision
// form instantiates them with float.
template <class T>
__device__ __forceinline__ void euler_flux(const T q[5], T F[3][5]) {
  const T rho = q[0], u = q[1], v = q[2], w = q[3], p = q[4];
  const T rs = fmax(rho, T(1e-10));
  const T ke = T(0.5) * (u * u + v * v + w * w);
  const T e_int = p / (T(GAMMA - 1.0) * rs);
  const T rhoE = rho * (e_int + ke);
  const T H = (rhoE + p) / rs;
  const T mf0 = rho * u, mf1 = rho * v, mf2 = rho * w;
  F[0][0] = mf0; F[0][1] = mf0 * u + p; F[0][2] = mf0 * v;     F[0][3] = mf0 * w;     F[0][4] = rho * H * u;
  F[1][0] = mf1; F[1][1] = mf1 * u;     F[1][2] = mf1 * v + p; F[1][3] = mf1 * w;     F[1][4] = rho * H * v;
  F[2][0] = mf2; F[2][1] = mf2 * u;     F[2][2] = mf2 * v;     F[2][3] = mf2 * w + p; F[2][4] = rho * H * w;
}

template <class T>
__device__ __forceinline__ T sq(T x) { return x * x; }

template <class T>
__device__ __forceinline__ void ausm_up(const T qL[5], const T qR[5], const T n[3], T out[5]) {
  const T alpha = T(0.1875), beta = T(0.5), Kp = T(0.25), Ku = T(0.75), sigma_p = T(1.0), ma_ref = T(0.1);
  const T rhoL = fmax(qL[0], T(1e-6)), rhoR = fmax(qR[0], T(1e-6));
  const T pL = fmax(qL[4], T(10.0)), pR = fmax(qR[4], T(10.0));
  const T uL = qL[1], vL = qL[2], wL = qL[3];
  const T uR = qR[1], vR = qR[2], wR = qR[3];
  const T unL = uL * n[0] + vL * n[1] + wL * n[2];
  const T unR = uR * n[0] + vR * n[1] + wR * n[2];
  const T aL = sqrt(fmax(T(GAMMA) * pL / rhoL, T(1e-10)));
  const T aR = sqrt(fmax(T(GAMMA) * pR / rhoR, T(1e-10)));
  const T ML = unL / fmax(aL, T(1e-10));
  const T MR = unR / fmax(aR, T(1e-10));
  const T a_half = T(0.5) * (aL + aR);
  const T rho_half = T(0.5) * (rhoL + rhoR);
  const T Mbar2 = (sq(unL) + sq(unR)) / (T(2.0) * sq(a_half));
  const T M0 = fmin(T(1.0), fmax(Mbar2, ma_ref * ma_ref));
  T fa = sqrt(M0) * (T(2.0) - sqrt(M0));
  fa = fmax(fa, T(1e-6));
  const T mp = (fabs(ML) >= T(1.0)) ? T(0.5) * (ML + fabs(ML)) : T(0.25) * sq(ML + T(1.0)) + alpha * sq(sq(ML) - T(1.0));
  const T mm = (fabs(MR) >= T(1.0)) ? T(0.5) * (MR - fabs(MR)) : -T(0.25) * sq(MR - T(1.0)) - alpha * sq(sq(MR) - T(1.0));
  const T M_half = mp + mm;
  const T Mp = -(Kp / fa) * fmax(T(1.0) - sigma_p * Mbar2, T(0.0)) * (pR - pL) / (rho_half * sq(a_half));
  const T mdot = T(0.5) * (rhoL * aL + rhoR * aR) * (M_half + Mp);
  const T sgnL = (ML > T(0.0)) ? T(1.0) : ((ML < T(0.0)) ? T(-1.0) : T(0.0));
  const T sgnR = (MR > T(0.0)) ? T(1.0) : ((MR < T(0.0)) ? T(-1.0) : T(0.0));
  const T PpL = (fabs(ML) >= T(1.0)) ? T(0.5) * (T(1.0) + sgnL)
                                     : T(0.25) * (sq(ML + T(1.0)) * (T(2.0) - ML) + beta * ML * sq(sq(ML) - T(1.0)));
  const T PmR = (fabs(MR) >= T(1.0)) ? T(0.5) * (T(1.0) - sgnR)
                                     : T(0.25) * (sq(MR - T(1.0)) * (T(2.0) + MR) - beta * MR * sq(sq(MR) - T(1.0)));
  const T p_half = PpL * pL + PmR * pR - Ku * PpL * PmR * (rhoL + rhoR) * fa * a_half * (unR - unL);
  const bool up = mdot >= T(0.0);
  out[0] = mdot;
  out[1] = mdot * (up ? uL : uR) + p_half * n[0];
  out[2] = mdot * (up ? vL : vR) + p_half * n[1];
  out[3] = mdot * (up ? wL : wR) + p_half * n[2];
  const T hL = T(GAMMA / (GAMMA - 1.0)) * pL / rhoL + T(0.5) * (sq(uL) + sq(vL) + sq(wL));
  const T hR = T(GAMMA / (GAMMA - 1.0)) * pR / rhoR + T(0.5) * (sq(uR) + sq(vR) + sq(wR));
  out[4] = mdot * (up ? hL : hR);
}

// gv[a*3+b] = d u_a / d x_b, gT[3], viscous flux G (3,5)
template <class T>
__device__ __forceinline__ void viscous_flux(const T q[5], const T gv[9], const T gT[3], T mu, T mu_t, T G[3][5]) {
  const T mt = mu + mu_t;
  const T S00 = gv[0], S11 = gv[4], S22 = gv[8];
  const T S01 = T(0.5) * (gv[1] + gv[3]);
  const T S02 = T(0.5) * (gv[2] + gv[6]);
  const T S12 = T(0.5) * (gv[5] + gv[7]);
  const T div = gv[0] + gv[4] + gv[8];
  const T lam = T(-2.0 / 3.0) * mt;
  const T t00 = T(2.0) * mt * S00 + lam * div;
  const T t11 = T(2.0) * mt * S11 + lam * div;
  const T t22 = T(2.0) * mt * S22 + lam * div;
  const T t01 = T(2.0) * mt * S01, t02 = T(2.0) * mt * S02, t12 = T(2.0) * mt * S12;
  const T cp = T(GAMMA * R_AIR / (GAMMA - 1.0));
  const T k = mu * cp / T(PR) + mu_t * cp / T(PR_T);
  const T u = q[1], v = q[2], w = q[3];
  G[0][0] = T(0.0); G[0][1] = t00; G[0][2] = t01; G[0][3] = t02;
  G[1][0] = T(0.0); G[1][1] = t01; G[1][2] = t11; G[1][3] = t12;
  G[2][0] = T(0.0); G[2][1] = t02; G[2][2] = t12; G[2][3] = t22;
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
template <class T>
__device__ __forceinline__ void ghost_state(const Bc& bc, int code, const T qo[5], const T n[3], T g[5]) {
  for (int v = 0; v < 5; ++v) g[v] = qo[v];
  const int t = bc.type[code];
  const T vn = qo[1] * n[0] + qo[2] * n[1] + qo[3] * n[2];
  if (t == BC_WALL) {
    if (bc.noslip[code]) {
      for (int d = 0; d < 3; ++d) g[1 + d] = T(2.0) * T(bc.wall_vel[code * 3 + d]) - qo[1 + d];
    } else {
      for (int d = 0; d < 3; ++d) g[1 + d] = qo[1 + d] - T(2.0) * vn * n[d];
    }
  } else if (t == BC_FARFIELD) {
    for (int v = 0; v < 5; ++v) g[v] = T(bc.Q[code * 5 + v]);
  } else if (t == BC_INLET) {
    if (vn < T(0.0))
      for (int v = 0; v < 5; ++v) g[v] = T(bc.Q[code * 5 + v]);
  } else if (t == BC_OUTLET) {
    if (vn > T(0.0)) g[4] = T(bc.p_out[code]);
  } else if (t == BC_SYMMETRY) {
    for (int d = 0; d < 3; ++d) g[1 + d] = qo[1 + d] - T(2.0) * vn * n[d];
  }
}

}  // namespace afr
