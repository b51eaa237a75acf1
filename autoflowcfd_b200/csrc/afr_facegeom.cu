// Flux-point construction on the device: for each face side that reads the
// other cell, locate the own face's flux points on the other cell's face and
// form the cross-interpolation rows from the other cell's solution points.
// Restates (paths relative to the reference's src/autoflowcfd):
//   build_fp_newton_parallel        fr/face_flux_points_numba.py:30-251
//   build_ms_interp_parallel        fr/face_flux_points_ms_numba.py:31-317
//   _face_ref_grid_nb, _map_*_nb    fr/face_flux_points_helpers_numba.py:53-124
//   _tet_exact_locate_nb            fr/face_flux_points_helpers_numba.py:134-197
//   _newton_locate_nb               fr/face_flux_points_helpers_numba.py:200-356
//   tet/prism_modal_basis_and_grad  fr/collapsed_basis.py:51-231 (values only)
//
// One warp per locate job, lane p = flux point p (at most 16).  The prism
// Newton iteration is coupled across the points of a face only through its
// stopping tests (maximum residual, "all improved / all steps small" of the
// line search); the warp evaluates those with votes and a max reduction, so
// every point takes exactly the reference's sequence of iterates.  The
// interpolation row of point p is V(p, :) * V_inv, summed over the modes in
// ascending order.  This file is compiled without multiply-add contraction so
// that every product and sum rounds as the reference's numpy / Numba code.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/afr_b200.h"

namespace {

constexpr int FP_MAX = 16, SPS_MAX = 64, N1D_MAX = 4, JOB_WARPS = 4;
constexpr int NEWTON_MAX_ITER = 50, LINE_SEARCH_MAX = 20;
__constant__ int c_face_axis[6] = {0, 0, 1, 1, 2, 2};
__constant__ double c_face_side[6] = {-1.0, 1.0, -1.0, 1.0, -1.0, 1.0};

struct FpGeom {
  int n_prism, n1d, n_fp, n_sps;
  const double* nodes;       // (n_nodes, 3)
  const int32_t* prism;      // (n_prism, 6)
  const int32_t* tet;        // (n_tet, 4)
  const double* vinv[2];     // prism, tet: (n_sps, n_sps), V_inv[m * n_sps + s]
  const double* sps;         // (n1d)
  const double* area;        // (n_faces)
  const double* trans;       // (n_faces, 3)
};

struct FpJobs {
  int n;
  const int32_t *face, *src_cell, *src_code, *tgt_cell, *tgt_code, *sign, *mode;
  const uint32_t* mask;
  double* mats;     // (n, n_fp, n_sps)
  double* coords;   // (n, n_fp, 2)
  double* resid;    // (n)
};

struct CellNodes {
  double x[6][3];
  bool prism;
};

__device__ void load_cell(const FpGeom& g, int c, CellNodes& cn) {
  cn.prism = c < g.n_prism;
  const int nv = cn.prism ? 6 : 4;
  const int32_t* ids = cn.prism ? g.prism + (size_t)c * 6 : g.tet + (size_t)(c - g.n_prism) * 4;
  for (int v = 0; v < nv; ++v)
    for (int d = 0; d < 3; ++d) cn.x[v][d] = g.nodes[(size_t)ids[v] * 3 + d];
}

// _map_prism_to_physical_nb / _map_tet_to_physical_nb at one reference point
__device__ void map_point(const CellNodes& cn, double a, double b, double c, double out[3]) {
  if (cn.prism) {
    const double s = b;
    const double r = (1.0 + a) * (1.0 - b) / 2.0 - 1.0;
    const double l1 = -(r + s) / 2.0, l2 = (1.0 + r) / 2.0, l3 = (1.0 + s) / 2.0;
    const double z = c;
    for (int d = 0; d < 3; ++d) {
      const double bottom = l1 * cn.x[0][d] + l2 * cn.x[1][d] + l3 * cn.x[2][d];
      const double top = l1 * cn.x[3][d] + l2 * cn.x[4][d] + l3 * cn.x[5][d];
      out[d] = 0.5 * (1.0 - z) * bottom + 0.5 * (1.0 + z) * top;
    }
  } else {
    const double t = c;
    const double s = (1.0 + b) * (1.0 - c) / 2.0 - 1.0;
    const double r = -(1.0 + a) * (s + t) / 2.0 - 1.0;
    const double L1 = -(1.0 + r + s + t) / 2.0, L2 = (1.0 + r) / 2.0, L3 = (1.0 + s) / 2.0, L4 = (1.0 + t) / 2.0;
    for (int d = 0; d < 3; ++d) out[d] = L1 * cn.x[0][d] + L2 * cn.x[1][d] + L3 * cn.x[2][d] + L4 * cn.x[3][d];
  }
}

// the two free axes of a face with fixed axis `ax`, ascending
__device__ __forceinline__ void free_axes(int ax, int& o0, int& o1) {
  o0 = ax == 0 ? 1 : 0;
  o1 = ax == 2 ? 1 : 2;
}

__device__ __forceinline__ void place(int ax, double side, double x0, double x1, double abc[3]) {
  int o0, o1;
  free_axes(ax, o0, o1);
  abc[ax] = side;
  abc[o0] = x0;
  abc[o1] = x1;
}

__device__ __forceinline__ double dist3(const double p[3], const double q[3]) {
  const double dx = p[0] - q[0], dy = p[1] - q[1], dz = p[2] - q[2];
  return sqrt(dx * dx + dy * dy + dz * dz);
}

__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// _tet_exact_locate_nb for one point (closed form on the face's vertices)
__device__ void tet_locate(const CellNodes& cn, int ax, double side, const double tgt[3], double& x0, double& x1) {
  int vi, vj, vk;
  if (ax == 0 && side < 0.0) { vi = 0; vj = 2; vk = 3; }
  else if (ax == 0 && side > 0.0) { vi = 1; vj = 2; vk = 3; }
  else if (ax == 1 && side < 0.0) { vi = 0; vj = 1; vk = 3; }
  else { vi = 0; vj = 1; vk = 2; }
  double e1[3], e2[3];
  for (int d = 0; d < 3; ++d) {
    e1[d] = cn.x[vj][d] - cn.x[vi][d];
    e2[d] = cn.x[vk][d] - cn.x[vi][d];
  }
  const double e1n = sqrt(fmax(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2], 1e-300));
  const double e2n = sqrt(fmax(e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2], 1e-300));
  double h1[3], h2[3];
  for (int d = 0; d < 3; ++d) {
    h1[d] = e1[d] / e1n;
    h2[d] = e2[d] / e2n;
  }
  const double a11 = h1[0] * h1[0] + h1[1] * h1[1] + h1[2] * h1[2];
  const double a12 = h1[0] * h2[0] + h1[1] * h2[1] + h1[2] * h2[2];
  const double a22 = h2[0] * h2[0] + h2[1] * h2[1] + h2[2] * h2[2];
  const double r0 = tgt[0] - cn.x[vi][0], r1 = tgt[1] - cn.x[vi][1], r2 = tgt[2] - cn.x[vi][2];
  const double b1 = r0 * h1[0] + r1 * h1[1] + r2 * h1[2];
  const double b2 = r0 * h2[0] + r1 * h2[1] + r2 * h2[2];
  const double det = a11 * a22 - a12 * a12;
  const double ds = fabs(det) > 1e-300 ? det : 1e-300;
  const double alpha = (b1 * a22 - b2 * a12) / ds / e1n;
  const double beta = (a11 * b2 - a12 * b1) / ds / e2n;
  double L[4] = {0.0, 0.0, 0.0, 0.0};
  L[vi] = 1.0 - alpha - beta;
  L[vj] = alpha;
  L[vk] = beta;
  const double r = 2.0 * L[1] - 1.0, s = 2.0 * L[2] - 1.0, t = 2.0 * L[3] - 1.0;
  const double cv = t;
  double db = 1.0 - cv;
  if (fabs(db) < 1e-300) db = 1e-300;
  const double bc = 2.0 * (s + 1.0) / db - 1.0;
  double da = s + t;
  if (fabs(da) < 1e-300) da = 1e-300;
  const double ac = -2.0 * (r + 1.0) / da - 1.0;
  const double full[3] = {ac, bc, cv};
  int o0, o1;
  free_axes(ax, o0, o1);
  x0 = full[o0];
  x1 = full[o1];
}

// residual |map(x) - target| of a point on the fixed face
__device__ __forceinline__ double point_resid(const CellNodes& cn, int ax, double side, double x0, double x1,
                                              const double tgt[3], double phys[3]) {
  double abc[3];
  place(ax, side, x0, x1, abc);
  map_point(cn, abc[0], abc[1], abc[2], phys);
  return dist3(phys, tgt);
}

// _newton_locate_nb for the lanes' points; returns the maximum residual
__device__ double locate(const CellNodes& cn, int ax, double side, const double tgt[3], bool act, double scale_in,
                         double& x0, double& x1) {
  const double scale = scale_in > 1e-300 ? scale_in : 1e-300;
  double phys[3];
  if (!cn.prism) {
    x0 = x1 = 0.0;
    double r = 0.0;
    if (act) {
      tet_locate(cn, ax, side, tgt, x0, x1);
      r = point_resid(cn, ax, side, x0, x1, tgt, phys);
    }
    return warp_max(r);
  }
  const double eps = 1e-6;
  x0 = x1 = 0.0;
  double rn = act ? point_resid(cn, ax, side, x0, x1, tgt, phys) : 0.0;
  double tol = 1e-13;
  if (1e-10 * scale > tol) tol = 1e-10 * scale;
  for (int it = 0; it < NEWTON_MAX_ITER; ++it) {
    if (warp_max(act ? rn : 0.0) < tol) break;
    double dx0 = 0.0, dx1 = 0.0;
    if (act) {
      double res[3], pp0[3], pp1[3];
      point_resid(cn, ax, side, x0, x1, tgt, phys);
      for (int d = 0; d < 3; ++d) res[d] = phys[d] - tgt[d];
      point_resid(cn, ax, side, x0 + eps, x1, tgt, pp0);
      point_resid(cn, ax, side, x0, x1 + eps, tgt, pp1);
      double J0[3], J1[3];
      for (int d = 0; d < 3; ++d) {
        J0[d] = (pp0[d] - phys[d]) / eps;
        J1[d] = (pp1[d] - phys[d]) / eps;
      }
      const double J0n = fmax(sqrt(J0[0] * J0[0] + J0[1] * J0[1] + J0[2] * J0[2]), 1e-300);
      const double J1n = fmax(sqrt(J1[0] * J1[0] + J1[1] * J1[1] + J1[2] * J1[2]), 1e-300);
      const double j00 = J0[0] / J0n, j01 = J0[1] / J0n, j02 = J0[2] / J0n;
      const double j10 = J1[0] / J1n, j11 = J1[1] / J1n, j12 = J1[2] / J1n;
      const double a11 = j00 * j00 + j01 * j01 + j02 * j02;
      const double a12 = j00 * j10 + j01 * j11 + j02 * j12;
      const double a22 = j10 * j10 + j11 * j11 + j12 * j12;
      const double b1 = -(j00 * res[0] + j01 * res[1] + j02 * res[2]);
      const double b2 = -(j10 * res[0] + j11 * res[1] + j12 * res[2]);
      const double det = a11 * a22 - a12 * a12;
      const double ds = fabs(det) > 1e-300 ? det : 1e-300;
      dx0 = (b1 * a22 - b2 * a12) / ds / J0n;
      dx1 = (a11 * b2 - a12 * b1) / ds / J1n;
    }
    // backtracking line search (the reference's two passes per round: the
    // second re-tests against the possibly improved best residual)
    double step = 1.0, xb0 = x0, xb1 = x1, rb = rn;
    for (int ls = 0; ls < LINE_SEARCH_MAX; ++ls) {
      bool imp = true, sml = true;
      if (act) {
        const double rt = point_resid(cn, ax, side, x0 + step * dx0, x1 + step * dx1, tgt, phys);
        if (rt < rb) {
          xb0 = x0 + step * dx0;
          xb1 = x1 + step * dx1;
          rb = rt;
        } else {
          imp = false;
        }
        if (step >= 1e-8) sml = false;
      }
      const bool all_imp = __all_sync(0xffffffffu, imp), all_sml = __all_sync(0xffffffffu, sml);
      if (all_imp || all_sml) break;
      if (act) {
        const double rt = point_resid(cn, ax, side, x0 + step * dx0, x1 + step * dx1, tgt, phys);
        if (!(rt < rb)) step *= 0.5;
      }
    }
    x0 = xb0;
    x1 = xb1;
    rn = rb;
  }
  return warp_max(act ? rn : 0.0);
}

// unnormalised Jacobi polynomial P_n^(alpha, beta)(x) by the three-term recurrence
__device__ double jacobi(double x, double alpha, double beta, int n) {
  double pm1 = 1.0;
  if (n == 0) return pm1;
  double p = 0.5 * ((alpha - beta) + (alpha + beta + 2.0) * x);
  if (n == 1) return p;
  for (int k = 1; k < n; ++k) {
    const double a1 = 2.0 * (k + 1) * (k + alpha + beta + 1) * (2 * k + alpha + beta);
    const double a2 = (2 * k + alpha + beta + 1) * (alpha * alpha - beta * beta);
    const double a3 = (2 * k + alpha + beta) * (2 * k + alpha + beta + 1) * (2 * k + alpha + beta + 2);
    const double a4 = 2.0 * (k + alpha) * (k + beta) * (2 * k + alpha + beta + 2);
    const double pn = ((a2 + a3 * x) * p - a4 * pm1) / a1;
    pm1 = p;
    p = pn;
  }
  return p;
}

// x**n for an integer n >= 0 by square-and-multiply from 1 (the rounding of
// the reference's compiled integer power)
__device__ __forceinline__ double ipow(double x, int n) {
  double r = 1.0, a = x;
  for (;;) {
    if (n & 1) r = r * a;
    n >>= 1;
    if (!n) break;
    a = a * a;
  }
  return r;
}

// modal basis values of point (a, b, c), modes flat = i*n1d^2 + j*n1d + k
__device__ void modal_row(bool prism, int n1d, double a, double b, double c, double* V) {
  const double h1b = (1.0 - b) / 2.0, h1c = (1.0 - c) / 2.0;
  for (int i = 0; i < n1d; ++i) {
    const double fi = jacobi(a, 0.0, 0.0, i);
    const double wi = i == 0 ? 1.0 : ipow(h1b, i);
    for (int j = 0; j < n1d; ++j) {
      const double g = fi * (wi * jacobi(b, (double)(2 * i + 1), 0.0, j));
      const int p = i + j;
      const double w = p == 0 ? 1.0 : ipow(h1c, p);
      for (int k = 0; k < n1d; ++k) {
        const int flat = (i * n1d + j) * n1d + k;
        if (prism) V[flat] = g * jacobi(c, 0.0, 0.0, k);
        else V[flat] = g * (w * jacobi(c, (double)(2 * i + 2 * j + 2), 0.0, k));
      }
    }
  }
}

__global__ void __launch_bounds__(32 * JOB_WARPS) k_flux_point_jobs(FpGeom g, FpJobs jb) {
  __shared__ double sV[JOB_WARPS][FP_MAX * SPS_MAX];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int job = blockIdx.x * JOB_WARPS + warp;
  if (job >= jb.n) return;  // whole warps leave together
  const int P = g.n_fp, S = g.n_sps, n1d = g.n1d;
  const int f = jb.face[job];
  const bool act = lane < P;
  CellNodes src, tgt;
  load_cell(g, jb.src_cell[job], src);
  load_cell(g, jb.tgt_cell[job], tgt);
  const int sax = c_face_axis[jb.src_code[job]], tax = c_face_axis[jb.tgt_code[job]];
  const double sside = c_face_side[jb.src_code[job]], tside = c_face_side[jb.tgt_code[job]];
  // the own face's flux point of this lane, mapped to physical space, and
  // the search target on the other side (periodic faces shift by the
  // face's translation: minus for owner -> neighbour, plus the other way)
  double target[3] = {0.0, 0.0, 0.0};
  if (act) {
    int o0, o1;
    free_axes(sax, o0, o1);
    double abc[3];
    abc[sax] = sside;
    abc[o0] = g.sps[lane / n1d];
    abc[o1] = g.sps[lane % n1d];
    map_point(src, abc[0], abc[1], abc[2], target);
    const double* t = g.trans + (size_t)f * 3;
    const bool ht = fabs(t[0]) > 1e-300 || fabs(t[1]) > 1e-300 || fabs(t[2]) > 1e-300;
    if (ht) {
      const double sg = jb.sign[job] > 0 ? 1.0 : -1.0;
      for (int d = 0; d < 3; ++d) target[d] = sg > 0.0 ? target[d] + t[d] : target[d] - t[d];
    }
  }
  const double cl = sqrt(fmax(g.area[f], 1e-300));
  double x0 = 0.0, x1 = 0.0;
  const double r = locate(tgt, tax, tside, target, act, cl, x0, x1);
  if (act) {
    jb.coords[((size_t)job * P + lane) * 2] = x0;
    jb.coords[((size_t)job * P + lane) * 2 + 1] = x1;
    double abc[3];
    place(tax, tside, x0, x1, abc);
    modal_row(tgt.prism, n1d, abc[0], abc[1], abc[2], &sV[warp][lane * S]);
  }
  if (lane == 0) jb.resid[job] = r;
  __syncwarp();
  // rows: V(p, :) * V_inv over the modes in ascending order; rows outside
  // the job's half of a split quad are zero
  const double* Vi = g.vinv[tgt.prism ? 0 : 1];
  const int mode = jb.mode[job];
  const uint32_t mask = jb.mask[job];
  double* out = jb.mats + (size_t)job * P * S;
  for (int p = 0; p < P; ++p) {
    const bool in = ((mask >> p) & 1u) != 0;
    const bool keep = mode == 0 || (mode == 1 && in) || (mode == 2 && !in);
    for (int s = lane; s < S; s += 32) {
      double val = 0.0;
      if (keep)
        for (int m = 0; m < S; ++m) val += sV[warp][p * S + m] * __ldg(Vi + (size_t)m * S + s);
      out[(size_t)p * S + s] = val;
    }
  }
}

template <class T>
cudaError_t dput(T** d, const T* h, size_t n, std::vector<void*>& owned) {
  *d = nullptr;
  if (n == 0) return cudaSuccess;
  cudaError_t e = cudaMalloc((void**)d, n * sizeof(T));
  if (e != cudaSuccess) return e;
  owned.push_back(*d);
  return h ? cudaMemcpy(*d, h, n * sizeof(T), cudaMemcpyHostToDevice) : cudaSuccess;
}

}  // namespace

extern "C" int afr_flux_point_jobs(int32_t order, int32_t n_prism, int64_t n_tet, int64_t n_nodes, const double* nodes,
                                   const int32_t* prism_conn, const int32_t* tet_conn, const double* v_inv_prism,
                                   const double* v_inv_tet, const double* sps_1d, int64_t n_faces, const double* area,
                                   const double* translation, int64_t n_jobs, const int32_t* face,
                                   const int32_t* src_cell, const int32_t* src_code, const int32_t* tgt_cell,
                                   const int32_t* tgt_code, const int32_t* sign, const int32_t* mode,
                                   const uint32_t* mask, double* mats, double* coords, double* resid) {
  if (order < 0 || order > 3 || n_prism < 0 || n_tet < 0 || n_nodes <= 0 || !nodes || n_faces <= 0 || !area ||
      !translation || n_jobs < 0 || !sps_1d)
    return AFR_EINVAL;
  if (n_jobs == 0) return AFR_OK;
  if (!face || !src_cell || !src_code || !tgt_cell || !tgt_code || !sign || !mode || !mask || !mats || !coords ||
      !resid)
    return AFR_EINVAL;
  if ((n_prism > 0 && (!prism_conn || !v_inv_prism)) || (n_tet > 0 && (!tet_conn || !v_inv_tet))) return AFR_EINVAL;
  const int n1d = order + 1, P = n1d * n1d, S = n1d * n1d * n1d;
  const int64_t n_cells = n_prism + n_tet;
  // every index in range before any kernel runs
  for (int64_t i = 0; i < (int64_t)n_prism * 6; ++i)
    if (prism_conn[i] < 0 || prism_conn[i] >= n_nodes) return AFR_EINDEX;
  for (int64_t i = 0; i < n_tet * 4; ++i)
    if (tet_conn[i] < 0 || tet_conn[i] >= n_nodes) return AFR_EINDEX;
  for (int64_t j = 0; j < n_jobs; ++j) {
    if (face[j] < 0 || face[j] >= n_faces || src_cell[j] < 0 || src_cell[j] >= n_cells || tgt_cell[j] < 0 ||
        tgt_cell[j] >= n_cells || src_code[j] < 0 || src_code[j] > 5 || tgt_code[j] < 0 || tgt_code[j] > 5 ||
        mode[j] < 0 || mode[j] > 2)
      return AFR_EINDEX;
  }
  std::vector<void*> owned;
  auto done = [&](int rc) {
    for (void* p : owned) cudaFree(p);
    return rc;
  };
  FpGeom g{};
  g.n_prism = n_prism;
  g.n1d = n1d;
  g.n_fp = P;
  g.n_sps = S;
  double *dn, *dvp, *dvt, *ds, *da, *dt;
  int32_t *dpc, *dtc;
  cudaError_t e = dput(&dn, nodes, (size_t)n_nodes * 3, owned);
  if (e == cudaSuccess) e = dput(&dpc, prism_conn, (size_t)n_prism * 6, owned);
  if (e == cudaSuccess) e = dput(&dtc, tet_conn, (size_t)n_tet * 4, owned);
  if (e == cudaSuccess) e = dput(&dvp, n_prism > 0 ? v_inv_prism : nullptr, n_prism > 0 ? (size_t)S * S : 0, owned);
  if (e == cudaSuccess) e = dput(&dvt, n_tet > 0 ? v_inv_tet : nullptr, n_tet > 0 ? (size_t)S * S : 0, owned);
  if (e == cudaSuccess) e = dput(&ds, sps_1d, (size_t)n1d, owned);
  if (e == cudaSuccess) e = dput(&da, area, (size_t)n_faces, owned);
  if (e == cudaSuccess) e = dput(&dt, translation, (size_t)n_faces * 3, owned);
  if (e != cudaSuccess) return done(AFR_ENOMEM);
  g.nodes = dn;
  g.prism = dpc;
  g.tet = dtc;
  g.vinv[0] = dvp;
  g.vinv[1] = dvt;
  g.sps = ds;
  g.area = da;
  g.trans = dt;
  // jobs in chunks that bound the device memory of the outputs
  const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(n_jobs, (int64_t)1 << 18));
  int32_t* dj[7];
  uint32_t* dm;
  double *dmats, *dcoords, *dres;
  for (int k = 0; k < 7 && e == cudaSuccess; ++k) e = dput(&dj[k], (const int32_t*)nullptr, (size_t)chunk, owned);
  if (e == cudaSuccess) e = dput(&dm, (const uint32_t*)nullptr, (size_t)chunk, owned);
  if (e == cudaSuccess) e = dput(&dmats, (const double*)nullptr, (size_t)chunk * P * S, owned);
  if (e == cudaSuccess) e = dput(&dcoords, (const double*)nullptr, (size_t)chunk * P * 2, owned);
  if (e == cudaSuccess) e = dput(&dres, (const double*)nullptr, (size_t)chunk, owned);
  if (e != cudaSuccess) return done(AFR_ENOMEM);
  const int32_t* hj[7] = {face, src_cell, src_code, tgt_cell, tgt_code, sign, mode};
  for (int64_t j0 = 0; j0 < n_jobs; j0 += chunk) {
    const int64_t n = std::min(chunk, n_jobs - j0);
    for (int k = 0; k < 7 && e == cudaSuccess; ++k)
      e = cudaMemcpy(dj[k], hj[k] + j0, n * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dm, mask + j0, n * sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return done(AFR_ECUDA);
    FpJobs jb{(int)n, dj[0], dj[1], dj[2], dj[3], dj[4], dj[5], dj[6], dm, dmats, dcoords, dres};
    k_flux_point_jobs<<<(unsigned)((n + JOB_WARPS - 1) / JOB_WARPS), 32 * JOB_WARPS>>>(g, jb);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(mats + (size_t)j0 * P * S, dmats, (size_t)n * P * S * sizeof(double),
                                         cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(coords + (size_t)j0 * P * 2, dcoords, (size_t)n * P * 2 * sizeof(double),
                                         cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(resid + j0, dres, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return done(AFR_ECUDA);
  }
  return done(AFR_OK);
}
