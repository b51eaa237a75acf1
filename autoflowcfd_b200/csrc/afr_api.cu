// C-ABI of the B200 FR residual-and-update library (declared in include/afr_b200.h).
//
// afr_create copies the reference's flattened mesh tables to HBM once, builds
// the per-cell slot lists (every face side that lifts a correction into a
// cell, in ascending face-color order) and allocates the scratch the step
// needs.  The step then runs, per RK stage, one gradient pre-pass and one
// fused per-cell stage kernel (see afr_kernels.cuh), plus the SST kernels once
// per step (afr_sst.cuh).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/afr_b200.h"
#include "afr_implicit.cuh"
#include "afr_mixed.cuh"
#include "afr_p0.cuh"
#include "afr_sst.cuh"

using namespace afr;

#define AFR_VERSION 100

struct afr_handle {
  int N = 0, n_prism = 0, order = 0, S = 0, Fn = 0, P = 0, F = 0, nv = 5;
  afr_params prm{};
  Geom g{};
  Ops ops{};
  Faces fc{};
  Bc bc{};
  // scratch
  double* PF = nullptr;       // (N,S,18) point fields of the state being evaluated
  double* J = nullptr;        // (n_slots,P,10) face jumps of the residual slots
  SlotTable slots{};
  double* Ua = nullptr;
  double* Ub = nullptr;
  double* dt = nullptr;
  double* norm_part = nullptr;
  double* norm_rho_part = nullptr;
  double* red = nullptr;      // reduction results
  double* red_part = nullptr; // per-chunk partials of the two-level reductions
  double* pt = nullptr;
  double* cfp = nullptr;
  double* sp8 = nullptr;
  uint8_t* wall_face = nullptr;
  uint8_t* cd_wall = nullptr;
  double* area_w = nullptr;
  int32_t* cd_faces = nullptr;
  int n_cd_faces = 0;
  double* cd_part = nullptr;  // (n_cd_faces, 6)
  unsigned* status = nullptr;
  // asynchronous status read of steps taken without a norm: the step copies
  // the device word into pinned host memory and records status_ev; the next
  // call on the handle reports a problem once that copy has completed
  unsigned* status_host = nullptr;
  cudaEvent_t status_ev = nullptr;
  bool status_pending = false;
  // order 0 (finite volume): face tables and per-face flux scratch
  P0Tab p0{};
  // mixed-precision form (prec == AFR_PREC_MIXED)
  int prec = AFR_PREC_FP64;
  MxOps mo{};
  MxFace mf{};
  MxBuf mb{};
  int mx_pre_blocks = 0, mx_cell_blocks = 0;  // resident CTAs of the persistent kernels
  int mx_pre_per_sm = 0, mx_pre_max_per_sm = 0, n_sms = 0;
  int mx_pre_occ = 0, mx_vol_occ = 0;          // occupancy-API CTAs per SM, before the tensor-memory cap
  // launch shapes chosen by afr_autotune (defaults until then)
  int mx_face_block = 128;  // threads per face-kernel CTA: 64, 128 or 256
  // matched interior face points paired across the face's two slots, and the
  // remaining slot points (boundary, interpolated, unpaired)
  int2* mx_pairs = nullptr;
  int32_t* mx_rest = nullptr;
  int mx_npairs = 0, mx_nrest = 0;
  bool mx_paired = false;
  int mx_upd_var = 1;       // update-kernel cells per CTA: 0 = half, 1 = base, 2 = double
  // dual-time / IMEX buffers, allocated by the first call of either scheme
  double* iRinv = nullptr;   // (N,S,nv) inviscid residual (dU/dt)
  double* iRvisc = nullptr;  // (N,S,nv) viscous residual (dU/dt)
  double* iRscr = nullptr;   // (N,S,nv) discarded inviscid residual of the IMEX iterations
  double* iUn = nullptr;     // (N,S,nv) state at the start of the physical step
  double* iX = nullptr;      // (N,S,nv) next iterate
  double* idt = nullptr;     // (N,S) physical time step of the dual-time SST update
  double* wprol = nullptr;   // (64 x 64) interpolation matrix of afr_prolong, allocated by its first call
  std::vector<void*> allocs;
  size_t mat_elems[4] = {0, 0, 0, 0};  // doubles of each interpolation-matrix allocation (0: shares the first)
  uint64_t bytes = 0;
  std::string err;
};

namespace {

thread_local std::string g_create_error;  // message of the last failed afr_create on this thread

int fail(afr_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

int cuda_fail(afr_handle* h, cudaError_t e, const char* what) {
  return fail(h, AFR_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
int dalloc(afr_handle* h, T** p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(h, AFR_ENOMEM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
  }
  h->allocs.push_back((void*)*p);
  h->bytes += n * sizeof(T);
  return AFR_OK;
}

template <class T>
int upload(afr_handle* h, T** dst, const T* src, size_t n, cudaStream_t st) {
  int rc = dalloc(h, dst, n);
  if (rc) return rc;
  if (src && n) {
    cudaError_t e = cudaMemcpyAsync(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(h, e, "upload");
  }
  return AFR_OK;
}

template <class T>
int upload_i32(afr_handle* h, int32_t** dst, const T* src, size_t n, cudaStream_t st, std::vector<int32_t>& tmp) {
  tmp.assign(n, 0);
  for (size_t i = 0; i < n; ++i) tmp[i] = (int32_t)src[i];
  int rc = upload(h, dst, tmp.data(), n, st);
  if (rc) return rc;
  cudaError_t e = cudaStreamSynchronize(st);  // tmp is reused by the caller
  return e == cudaSuccess ? AFR_OK : cuda_fail(h, e, "upload sync");
}

__global__ void k_form_adj(const double* det, const double* inv, double* adj, size_t npts) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * 9) return;
  adj[t] = det[t / 9] * inv[t];  // compute_adj_j, core/fr_operators/volume_contract.py:47-80
}

// |volume|^(1/3) per cell, the length of the local time step (core/fr_solver/cfl.py)
__global__ void k_cube_root_abs(const double* v, size_t n, double* out) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = pow(fabs(v[t]), 1.0 / 3.0);
}

__global__ void k_metric_flux_scale(const double* adj, double* mfs, size_t npts) {
  const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const double* a = adj + p * 9;
  double acc = 0.0;  // sum_m |adj[m,:]|, core/fr_solver/solver_geometry.py:18-32
  for (int m = 0; m < 3; ++m) acc += sqrt(a[m * 3] * a[m * 3] + a[m * 3 + 1] * a[m * 3 + 1] + a[m * 3 + 2] * a[m * 3 + 2]);
  mfs[p] = acc;
}

// deterministic single-block reductions (fixed order for a given n)
__global__ void k_reduce_sum(const double* x, size_t n, double* out) {
  __shared__ double sh[1024];
  double acc = 0.0;
  for (size_t i = threadIdx.x; i < n; i += blockDim.x) acc += x[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

// First level of the deterministic reductions: CTA b sums (or takes the
// minimum of) x[b*RED_CHUNK, (b+1)*RED_CHUNK) in a fixed order; the second
// level runs k_reduce_sum / k_reduce_min over the partials in one CTA.
constexpr int RED_CHUNK = 8192, RED_THREADS = 256;
template <bool MIN>
__global__ void __launch_bounds__(RED_THREADS) k_reduce_chunks(const double* __restrict__ x, size_t n,
                                                               double* __restrict__ part) {
  __shared__ double sh[RED_THREADS];
  const size_t b0 = (size_t)blockIdx.x * RED_CHUNK, b1 = b0 + RED_CHUNK < n ? b0 + RED_CHUNK : n;
  double acc = MIN ? INFINITY : 0.0;
  for (size_t i = b0 + threadIdx.x; i < b1; i += RED_THREADS) acc = MIN ? fmin(acc, x[i]) : acc + x[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = RED_THREADS / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] = MIN ? fmin(sh[threadIdx.x], sh[threadIdx.x + o]) : sh[threadIdx.x] + sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_reduce_min(const double* x, size_t n, double* out) {
  __shared__ double sh[1024];
  double acc = INFINITY;
  for (size_t i = threadIdx.x; i < n; i += blockDim.x) acc = fmin(acc, x[i]);
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] = fmin(sh[threadIdx.x], sh[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

__global__ void k_fill_value(double* x, size_t n, double v) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = v;
}

__global__ void k_fill_scaled(double* x, size_t n, const double* v, double factor) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = factor * (*v);
}

// per wall face: pressure and viscous force partials (postprocess/fr_coefficients.py:105-133)
template <int S, int NP>
__global__ void k_force(Geom g, Ops ops, Faces fc, const int32_t* faces, int nf, const double* U, int nv,
                        const double* PF, const double* nut, const double* area_w, double mu, double* part) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nf) return;
  const int f = faces[t];
  const int oc = fc.owner[f];
  const int ct = cell_type(g, oc);
  const int ax = fc.o_axis[f];
  const double* E = ops.extrap + (((size_t)ct * 3 + ax) * 2 + (fc.o_side[f] < 0.0 ? 0 : 1)) * NP * S;
  double fp[3] = {0, 0, 0}, fv[3] = {0, 0, 0};
  for (int i = 0; i < NP; ++i) {
    double pf = 0.0, mt = 0.0, gv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int s = 0; s < S; ++s) {
      const size_t p = (size_t)oc * S + s;
      const double* u = U + p * nv;
      const double rho = fmax(u[0], 1e-10);
      const double ux = u[1] / rho, uy = u[2] / rho, uz = u[3] / rho;
      const double pr = fmax((u[4] - rho * (0.5 * (ux * ux + uy * uy + uz * uz))) * 0.4, 1.0);
      const double w = E[i * S + s];
      pf += w * pr;
      if (nut) mt += w * (rho * nut[p]);
      for (int k = 0; k < 9; ++k) gv[k] += w * PF[p * PFW + 5 + k];
    }
    const double* n = fc.tnormal + ((size_t)f * NP + i) * 3;
    const double aw = area_w[(size_t)f * NP + i];
    for (int d = 0; d < 3; ++d) fp[d] += pf * n[d] * aw;
    const double mtot = mu + mt;
    const double div = gv[0] + gv[4] + gv[8];
    for (int r = 0; r < 3; ++r) {
      double tr = 0.0;
      for (int c = 0; c < 3; ++c) {
        const double sij = 0.5 * (gv[r * 3 + c] + gv[c * 3 + r]);
        const double tau = 2.0 * mtot * sij + ((r == c) ? (-2.0 / 3.0 * mtot) * div : 0.0);
        tr += tau * n[c];
      }
      fv[r] += tr * aw;
    }
  }
  for (int d = 0; d < 3; ++d) {
    part[t * 6 + d] = fp[d];
    part[t * 6 + 3 + d] = fv[d];
  }
}

// Optional event recorder for afr_step_profile: an event after every launch group.
struct StepTimer {
  cudaEvent_t ev[24];
  int n = 0;
  void mark(cudaStream_t st) {
    if (n < 24) cudaEventRecord(ev[n++], st);
  }
};

// n matrices (P, S) row-major -> (S, P) each (face point fastest on the device)
static std::vector<double> transpose_mats(const double* src, size_t n, int P, int S) {
  std::vector<double> out(n * P * S);
  for (size_t k = 0; k < n; ++k)
    for (int i = 0; i < P; ++i)
      for (int s = 0; s < S; ++s) out[(k * S + s) * P + i] = src[(k * P + i) * S + s];
  return out;
}

// CTAs of a kernel that fit on one SM by registers (allocated per warp in
// units of 256), shared memory (static + dynamic + the per-CTA reservation),
// threads and the CTA limit
static cudaError_t resident_ctas(const void* fn, int threads, size_t dyn_smem, int dev, int* out) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, fn);
  int smem_sm = 0, regs_sm = 0, thr_sm = 0, blk_sm = 0, resv = 0;
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&blk_sm, cudaDevAttrMaxBlocksPerMultiprocessor, dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock, dev);
  if (e != cudaSuccess) return e;
  const long warps = (threads + 31) / 32;
  const long regs_cta = warps * (((long)fa.numRegs * 32 + 255) / 256 * 256);
  const size_t smem_cta = fa.sharedSizeBytes + dyn_smem + (size_t)resv;
  long n = blk_sm;
  if (regs_cta > 0) n = std::min(n, (long)regs_sm / regs_cta);
  n = std::min(n, (long)(smem_sm / smem_cta));
  n = std::min(n, (long)thr_sm / (warps * 32));
  *out = (int)n;
  return cudaSuccess;
}

// SST source, transport and point-implicit update of one step (the three
// per-step kernels); cells of each type in their own launches
template <int S, int NP>
cudaError_t sst_launch(afr_handle* h, const SstArgs& a, cudaStream_t st, StepTimer* tm) {
  constexpr int CPB = SstTile<S>::CPB, TH = SstTile<S>::THREADS;
  const int ranges[3] = {0, h->n_prism, h->N};
  for (int r = 0; r < 2; ++r) {
    const int n = ranges[r + 1] - ranges[r];
    if (n > 0) k_sst_point<S><<<(n + CPB - 1) / CPB, TH, 0, st>>>(h->g, h->ops, a, ranges[r], ranges[r + 1]);
  }
  if (tm) tm->mark(st);
  if (h->F > 0)
    k_sst_face<S, NP><<<(h->F + SST_FACE_WARPS - 1) / SST_FACE_WARPS, 32 * SST_FACE_WARPS, 0, st>>>(h->g, h->ops,
                                                                                                    h->fc, a);
  if (tm) tm->mark(st);
  for (int r = 0; r < 2; ++r) {
    const int n = ranges[r + 1] - ranges[r];
    if (n > 0)
      k_sst_update<S, NP><<<(n + CPB - 1) / CPB, TH, 0, st>>>(h->g, h->ops, h->fc, a, ranges[r], ranges[r + 1]);
  }
  if (tm) tm->mark(st);
  return cudaGetLastError();
}

template <int S, int FN, int NP, int N1D>
struct Launch {
  static constexpr int CPB = S <= 8 ? 8 : (S <= 27 ? 2 : 1);
  static size_t cell_smem() { return sizeof(double) * CellSmem<S, FN, CPB, NP>::total; }
  static cudaError_t pre(afr_handle* h, const double* U, const double* nut, bool grads, cudaStream_t st) {
    constexpr int CPB = PreTile<S>::CPB;
    const int ranges[3] = {0, h->n_prism, h->N};
    for (int r = 0; r < 2; ++r) {
      const int n = ranges[r + 1] - ranges[r];
      if (n > 0)
        k_pre<S><<<(n + CPB - 1) / CPB, 128, 0, st>>>(h->g, h->ops, U, h->nv, nut, grads ? 1 : 0, h->PF, ranges[r],
                                                      ranges[r + 1]);
    }
    return cudaGetLastError();
  }
  static cudaError_t stage(afr_handle* h, StageArgs a, cudaStream_t st, StepTimer* tm = nullptr) {
    constexpr int SPW = 32 / NP;  // slots per warp of the face kernel
    const int nwarps = (h->slots.n + SPW - 1) / SPW;
    if (nwarps > 0)
      k_face<S, NP><<<(nwarps + FACE_WARPS - 1) / FACE_WARPS, 32 * FACE_WARPS, 0, st>>>(
          h->g, h->ops, h->fc, h->bc, h->slots, h->PF, h->prm.mu, a.inviscid_only ? 0 : 1, h->J);
    if (tm) tm->mark(st);
    const size_t smem = cell_smem();
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(k_cell<S, FN, NP, CPB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      attr = true;
    }
    a.N = h->N;
    a.slot_flags = h->slots.flags;
    const int ranges[3] = {0, h->n_prism, h->N};
    for (int r = 0; r < 2; ++r) {
      a.cell_base = ranges[r];
      a.cell_end = ranges[r + 1];
      const int n = a.cell_end - a.cell_base;
      if (n <= 0) continue;
      k_cell<S, FN, NP, CPB><<<(n + CPB - 1) / CPB, CELL_THREADS, smem, st>>>(h->g, h->ops, h->fc, a, h->J);
    }
    return cudaGetLastError();
  }
  // ---- mixed-precision form ----
  static constexpr int MXC = 16;                            // cells per volume-kernel tile
  static constexpr int MXU = S <= 8 ? 16 : (S <= 27 ? 4 : 2);  // cells per update-kernel CTA
  static size_t mx_pre_smem() { return MxPreSmem<S, NP>::total; }
  static size_t mx_vol_smem() { return MxVolSmem<S, FN, MXC>::total; }
  static constexpr int MXU0 = MXU / 2 > 0 ? MXU / 2 : 1, MXU2 = MXU * 2;  // autotuner candidates
  static size_t mx_upd_smem() { return MxUpdSmem<S, NP, MXU>::total; }
  // resident CTAs per SM of the persistent kernels, capped by tensor memory (512 columns per SM)
  static cudaError_t mx_grids(afr_handle* h) {
    int dev = 0, sms = 0, bp = 0, bc = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_mx_pre<S, NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx_pre_smem());
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_mx_vol<S, FN, MXC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx_vol_smem());
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_mx_update<S, NP, MXU>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)mx_upd_smem());
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_mx_update<S, NP, MXU0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)MxUpdSmem<S, NP, MXU0>::total);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_mx_update<S, NP, MXU2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)MxUpdSmem<S, NP, MXU2>::total);
    // the largest shared-memory carveout for the two persistent kernels, whose
    // shared memory sets how many CTAs fit on an SM
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_mx_pre<S, NP>, cudaFuncAttributePreferredSharedMemoryCarveout,
                               (int)cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_mx_vol<S, FN, MXC>, cudaFuncAttributePreferredSharedMemoryCarveout,
                               (int)cudaSharedmemCarveoutMaxShared);

    // The runtime's occupancy query answers one CTA per SM for every kernel
    // that uses tensor memory (it cannot know the allocation size), while the
    // SM co-schedules more where registers, shared memory and threads allow:
    // the residency is computed from those here and capped by the columns.
    int api_p = 0, api_c = 0;
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&api_p, k_mx_pre<S, NP>, MX_THREADS, mx_pre_smem());
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&api_c, k_mx_vol<S, FN, MXC>, MX_VOL_THREADS, mx_vol_smem());
    if (e == cudaSuccess) e = resident_ctas((const void*)k_mx_pre<S, NP>, MX_THREADS, mx_pre_smem(), dev, &bp);
    if (e == cudaSuccess) e = resident_ctas((const void*)k_mx_vol<S, FN, MXC>, MX_VOL_THREADS, mx_vol_smem(), dev, &bc);
    if (e != cudaSuccess) return e;
    h->mx_pre_occ = api_p;
    h->mx_vol_occ = api_c;
    bp = std::min(bp, 512 / MxPreSmem<S, NP>::NCOL);
    bc = std::min(bc, 512 / MxVolSmem<S, FN, MXC>::NCOL);
    if (bp < 1 || bc < 1) return cudaErrorInvalidConfiguration;
    h->mx_pre_blocks = bp * sms;
    h->mx_cell_blocks = bc * sms;
    h->mx_pre_per_sm = h->mx_pre_max_per_sm = bp;
    h->n_sms = sms;
    return cudaSuccess;
  }
  template <int CPB>
  static void mx_update_launch(afr_handle* h, const StageArgs& a, int n, cudaStream_t st) {
    k_mx_update<S, NP, CPB><<<(n + CPB - 1) / CPB, MxUpdSmem<S, NP, CPB>::THREADS, MxUpdSmem<S, NP, CPB>::total, st>>>(
        h->g, h->ops, h->fc, a, h->mb.RV, h->mb.Jm, h->mo.rdet);
  }
  static int n_ranges(const afr_handle* h) { return (h->n_prism > 0 ? 1 : 0) + (h->N > h->n_prism ? 1 : 0); }
  static cudaError_t mx_pre(afr_handle* h, const double* U, const double* nut, bool grads, cudaStream_t st) {
    const int ranges[3] = {0, h->n_prism, h->N};
    for (int r = 0; r < 2; ++r) {
      const int n = ranges[r + 1] - ranges[r];
      if (n <= 0) continue;
      const int tiles = (n + MX_PRE_CELLS - 1) / MX_PRE_CELLS;
      k_mx_pre<S, NP><<<std::min(tiles, h->mx_pre_blocks), MX_THREADS, mx_pre_smem(), st>>>(
          h->g, h->mo, h->mb, U, h->nv, nut, grads ? 1 : 0, ranges[r], ranges[r + 1], h->status);
    }
    return cudaGetLastError();
  }
  static cudaError_t mx_stage(afr_handle* h, StageArgs a, cudaStream_t st, StepTimer* tm) {
    const int nt = h->slots.n * NP;
    const int fb = h->mx_face_block;
    if (h->mx_paired) {
      if (h->mx_npairs > 0)
        k_mx_face_pair<S, NP><<<(h->mx_npairs + fb - 1) / fb, fb, 0, st>>>(
            h->fc, h->bc, h->slots, h->mf, h->mb, h->mo.hcell, (float)h->prm.mu, a.inviscid_only ? 0 : 1,
            h->mx_pairs, h->mx_npairs);
      if (h->mx_nrest > 0)
        k_mx_face<S, NP><<<(h->mx_nrest + fb - 1) / fb, fb, 0, st>>>(
            h->fc, h->bc, h->slots, h->mf, h->mb, h->mo.hcell, (float)h->prm.mu, a.inviscid_only ? 0 : 1,
            h->mx_rest, h->mx_nrest);
    } else if (nt > 0) {
      k_mx_face<S, NP><<<(nt + fb - 1) / fb, fb, 0, st>>>(h->fc, h->bc, h->slots, h->mf, h->mb, h->mo.hcell,
                                                           (float)h->prm.mu, a.inviscid_only ? 0 : 1, nullptr, 0);
    }
    if (tm) tm->mark(st);
    const int ranges[3] = {0, h->n_prism, h->N};
    for (int r = 0; r < 2; ++r) {
      const int n = ranges[r + 1] - ranges[r];
      if (n <= 0) continue;
      const int tiles = (n + MXC - 1) / MXC;
      k_mx_vol<S, FN, MXC><<<std::min(tiles, h->mx_cell_blocks), MX_VOL_THREADS, mx_vol_smem(), st>>>(
          h->g, h->mo, a.Ucur, h->nv, a.inviscid_only, (float)h->prm.mu, h->mb.PFm, h->mb.RV, ranges[r],
          ranges[r + 1], h->status);
    }
    if (tm) tm->mark(st);
    a.N = h->N;
    a.slot_flags = h->slots.flags;
    for (int r = 0; r < 2; ++r) {
      a.cell_base = ranges[r];
      a.cell_end = ranges[r + 1];
      const int n = a.cell_end - a.cell_base;
      if (n <= 0) continue;
      if (h->mx_upd_var == 0) mx_update_launch<MXU0>(h, a, n, st);
      else if (h->mx_upd_var == 2) mx_update_launch<MXU2>(h, a, n, st);
      else mx_update_launch<MXU>(h, a, n, st);
    }
    return cudaGetLastError();
  }
  // one residual evaluation of either form: pre-pass, face kernel, cell kernel;
  // adds the number of kernel launches to *nl
  static cudaError_t eval(afr_handle* h, StageArgs a, const double* U, const double* nut, bool grads,
                          cudaStream_t st, StepTimer* tm = nullptr, int* nl = nullptr) {
    const bool mx = h->prec == AFR_PREC_MIXED;
    cudaError_t r = mx ? mx_pre(h, U, nut, grads, st) : pre(h, U, nut, grads, st);
    if (r != cudaSuccess) return r;
    if (tm) tm->mark(st);
    if (nl) *nl += (mx ? n_ranges(h) : 1) + (h->slots.n > 0 ? 1 : 0) + (mx ? 2 : 1) * n_ranges(h);
    if (mx) return mx_stage(h, a, st, tm);
    r = stage(h, a, st, tm);
    if (tm) tm->mark(st);  // the plain form has no separate update kernel: an empty interval
    return r;
  }
  static cudaError_t sst(afr_handle* h, const SstArgs& a, cudaStream_t st, StepTimer* tm = nullptr) {
    return sst_launch<S, NP>(h, a, st, tm);
  }
  static cudaError_t force(afr_handle* h, const double* U, const double* nut, cudaStream_t st) {
    if (h->n_cd_faces == 0) return cudaSuccess;
    k_force<S, NP><<<(h->n_cd_faces + 127) / 128, 128, 0, st>>>(h->g, h->ops, h->fc, h->cd_faces, h->n_cd_faces, U,
                                                                 h->nv, h->PF, nut, h->area_w, h->prm.mu,
                                                                 h->cd_part);
    return cudaGetLastError();
  }
};

// Order 0: the finite-volume face kernel and the per-cell gather-and-update
// kernel stand in for the three kernels of a stage.  Gradients (the force
// integral's pre-pass) use the generic one-point kernels.
struct LaunchP0 {
  static cudaError_t pre(afr_handle* h, const double* U, const double* nut, bool grads, cudaStream_t st) {
    constexpr int CPB = PreTile<1>::CPB;
    const int ranges[3] = {0, h->n_prism, h->N};
    for (int r = 0; r < 2; ++r) {
      const int n = ranges[r + 1] - ranges[r];
      if (n > 0)
        k_pre<1><<<(n + CPB - 1) / CPB, 128, 0, st>>>(h->g, h->ops, U, h->nv, nut, grads ? 1 : 0, h->PF, ranges[r],
                                                      ranges[r + 1]);
    }
    return cudaGetLastError();
  }
  static cudaError_t eval(afr_handle* h, StageArgs a, const double* U, const double* nut, bool grads,
                          cudaStream_t st, StepTimer* tm = nullptr, int* nl = nullptr) {
    (void)grads;
    if (tm) tm->mark(st);  // no pre-pass: an empty interval
    k_p0_face<<<(h->F + 127) / 128, 128, 0, st>>>(h->g, h->fc, h->bc, h->p0, U, h->nv, nut, h->prm.mu,
                                                  a.inviscid_only ? 0 : 1);
    if (tm) tm->mark(st);
    a.N = h->N;
    k_p0_cell<<<(h->N + 127) / 128, 128, 0, st>>>(h->g, h->ops, h->fc, h->p0, a);
    if (tm) tm->mark(st);
    if (nl) *nl += 2;
    return cudaGetLastError();
  }
  // SST at one point per cell: the generic kernels with S = P = 1 (the
  // reference runs its FR transport and closure there, not a finite-volume form)
  static cudaError_t sst(afr_handle* h, const SstArgs& a, cudaStream_t st, StepTimer* tm = nullptr) {
    return sst_launch<1, 1>(h, a, st, tm);
  }
  static cudaError_t force(afr_handle* h, const double* U, const double* nut, cudaStream_t st) {
    if (h->n_cd_faces == 0) return cudaSuccess;
    k_force<1, 1><<<(h->n_cd_faces + 127) / 128, 128, 0, st>>>(h->g, h->ops, h->fc, h->cd_faces, h->n_cd_faces, U,
                                                               h->nv, h->PF, nut, h->area_w, h->prm.mu, h->cd_part);
    return cudaGetLastError();
  }
  static cudaError_t mx_grids(afr_handle*) { return cudaErrorNotSupported; }  // refused at create
};

// ---- host-side BF16 hi+lo operator images for the mixed form ----
uint16_t bf16_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u += 0x7fffu + ((u >> 16) & 1u);  // round to nearest even (operators are finite)
  return (uint16_t)(u >> 16);
}
float bf16_value(uint16_t b) {
  const uint32_t u = (uint32_t)b << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}
// R x K matrix -> [hi | lo] images in the K-major canonical layout
template <class Get>
std::vector<uint16_t> kmajor_image(int R, int K, Get get) {
  std::vector<uint16_t> img(2 * (size_t)R * K, 0);
  for (int r = 0; r < R; ++r)
    for (int k = 0; k < K; ++k) {
      const double x = get(r, k);
      const uint16_t hi = bf16_bits((float)x);
      const uint16_t lo = bf16_bits((float)(x - (double)bf16_value(hi)));
      const size_t idx = ((size_t)(k >> 3) * R + r) * 8 + (k & 7);
      img[idx] = hi;
      img[(size_t)R * K + idx] = lo;
    }
  return img;
}

// N x K matrix -> one stacked image of 2N rows: the hi parts over the lo parts
template <class Get>
std::vector<uint16_t> kmajor_image_cat(int N, int K, Get get) {
  auto split = kmajor_image(N, K, get);  // [hi | lo], each N x K
  std::vector<uint16_t> img(2 * (size_t)N * K, 0);
  for (int r = 0; r < N; ++r)
    for (int k = 0; k < K; ++k) {
      const size_t src = ((size_t)(k >> 3) * N + r) * 8 + (k & 7);
      img[((size_t)(k >> 3) * 2 * N + r) * 8 + (k & 7)] = split[src];
      img[((size_t)(k >> 3) * 2 * N + N + r) * 8 + (k & 7)] = split[(size_t)N * K + src];
    }
  return img;
}

template <class Fn>
cudaError_t dispatch(afr_handle* h, Fn&& fn) {
  switch (h->order) {
    case 0: return fn(LaunchP0());
    case 1: return fn(Launch<8, 27, 4, 2>());
    case 2: return fn(Launch<27, 64, 9, 3>());
    case 3: return fn(Launch<64, 64, 16, 4>());
  }
  return cudaErrorInvalidValue;
}

int status_code(afr_handle* h, unsigned s) {
  if (s & DS_BAD_INDEX) return fail(h, AFR_EINDEX, "kernel saw an out-of-range table index");
  if (s & DS_NONFINITE) return fail(h, AFR_ENONFINITE, "non-finite value in the state");
  if (s & DS_TC_TIMEOUT) return fail(h, AFR_ECUDA, "a tensor-core completion wait timed out");
  return AFR_OK;
}

int check_status(afr_handle* h, cudaStream_t st) {
  unsigned s = 0;
  cudaError_t e = cudaMemcpyAsync(&s, h->status, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(h, e, "status read");
  h->status_pending = false;
  return status_code(h, s);
}

bool capturing(cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  return cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone;
}

// Status of an earlier step taken without a norm, if its asynchronous copy has
// completed; never waits.
int pending_status(afr_handle* h, cudaStream_t st) {
  if (!h->status_pending || capturing(st)) return AFR_OK;
  const cudaError_t q = cudaEventQuery(h->status_ev);
  if (q == cudaErrorNotReady) {
    (void)cudaGetLastError();  // not an error: leave no trace for later launch checks
    return AFR_OK;
  }
  if (q != cudaSuccess) return cuda_fail(h, q, "status event");
  h->status_pending = false;
  return status_code(h, *h->status_host);
}

// Queue the copy of the device status word to the pinned host word.  Outside
// stream capture an event marks its completion for pending_status; inside a
// capture the copy becomes part of the graph and afr_status reads the word.
cudaError_t queue_status_copy(afr_handle* h, cudaStream_t st) {
  cudaError_t e = cudaMemcpyAsync(h->status_host, h->status, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess || capturing(st)) return e;
  e = cudaEventRecord(h->status_ev, st);
  if (e == cudaSuccess) h->status_pending = true;
  return e;
}

StageArgs base_args(afr_handle* h) {
  StageArgs a{};
  a.N = h->N;
  a.nv = h->nv;
  a.mu = h->prm.mu;
  a.inviscid_only = h->prm.inviscid_only;
  a.status = h->status;
  a.PF = h->PF;
  return a;
}

int compute_dt(afr_handle* h, const double* U, const double* nut, double* dt, cudaStream_t st) {
  const size_t n = (size_t)h->N * h->S;
  k_local_dt<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(h->g, h->S, h->order, U, h->nv, nut, h->prm.mu, dt);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(h, e, "local dt");
  if (h->prm.global_dt_factor > 0.0) {
    const unsigned nb = (unsigned)((n + RED_CHUNK - 1) / RED_CHUNK);
    k_reduce_chunks<true><<<nb, RED_THREADS, 0, st>>>(dt, n, h->red_part);
    k_reduce_min<<<1, 1024, 0, st>>>(h->red_part, nb, h->red);
    k_fill_scaled<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(dt, n, h->red, h->prm.global_dt_factor);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(h, e, "global dt");
  }
  return AFR_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// Allocation-free RMS norm.  Its per-block partial sums live in a fixed
// file-scope device array instead of handle scratch, so the call needs no
// cudaMalloc.  Every GPU that loads the library keeps these 32 KiB until exit.
// ---------------------------------------------------------------------------
constexpr int NOALLOC_PARTIALS = 4096;         // blocks, one partial each
constexpr int NOALLOC_THREADS = 256;
constexpr int64_t NOALLOC_CHUNK = 65536;       // elements summed per block
static __device__ __align__(256) double g_noalloc_partials[NOALLOC_PARTIALS];

namespace {
std::mutex g_noalloc_mutex;
double* g_noalloc_ptr[256] = {nullptr};        // per device ordinal

__global__ void k_sumsq_chunks(const double* __restrict__ x, int64_t n, double* __restrict__ partials) {
  __shared__ double sh[NOALLOC_THREADS];
  const int64_t beg = (int64_t)blockIdx.x * NOALLOC_CHUNK;
  const int64_t end = min(beg + NOALLOC_CHUNK, n);
  double acc = 0.0;
  for (int64_t i = beg + threadIdx.x; i < end; i += NOALLOC_THREADS) acc += x[i] * x[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = NOALLOC_THREADS / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = sh[0];
}

__global__ void k_rms_finish(const double* __restrict__ partials, int nb, int64_t n, double* out) {
  __shared__ double sh[1024];
  double acc = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) acc += partials[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = n > 0 ? sqrt(sh[0]) / sqrt((double)n) : 0.0;
}
}  // namespace

extern "C" {

int afr_rms_norm_noalloc(const double* x, int64_t n, double* out, void* stream) {
  if (n < 0 || !out || (n > 0 && !x)) return AFR_EINVAL;
  if (n > (int64_t)NOALLOC_PARTIALS * NOALLOC_CHUNK) return AFR_EINVAL;  // beyond the fixed scratch
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return AFR_ECUDA;
  double* partials = nullptr;
  {
    // once per device, with that device current: the device address of the
    // static array (its host-side name is only a stand-in)
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
      if (cudaGetSymbolAddress((void**)&g_noalloc_ptr[dev], g_noalloc_partials) != cudaSuccess) {
        g_noalloc_ptr[dev] = nullptr;
        return AFR_ECUDA;
      }
    }
    partials = g_noalloc_ptr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = (int)((n + NOALLOC_CHUNK - 1) / NOALLOC_CHUNK);
  if (nb > 0) k_sumsq_chunks<<<nb, NOALLOC_THREADS, 0, st>>>(x, n, partials);
  k_rms_finish<<<1, 1024, 0, st>>>(partials, nb, n, out);
  return cudaGetLastError() == cudaSuccess ? AFR_OK : AFR_ECUDA;
}

int afr_version(void) { return AFR_VERSION; }

const char* afr_status_string(int s) {
  switch (s) {
    case AFR_OK: return "ok";
    case AFR_EINVAL: return "invalid argument";
    case AFR_ENOMEM: return "out of device memory";
    case AFR_ECUDA: return "CUDA error";
    case AFR_ENONFINITE: return "non-finite value";
    case AFR_EUNSUPPORTED: return "unsupported";
    case AFR_EINDEX: return "index out of range";
  }
  return "unknown status";
}

const char* afr_last_error(const afr_handle* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int afr_greedy_face_coloring(int64_t n_faces, int64_t n_cells, const int64_t* owner, const int64_t* neighbor,
                             const uint8_t* is_boundary, int32_t* colors) {
  if (n_faces < 0 || n_cells < 0 || !owner || !neighbor || !is_boundary || !colors) return AFR_EINVAL;
  // cell -> faces touching it (owner always, neighbour of interior faces)
  std::vector<int64_t> cnt(n_cells + 1, 0);
  for (int64_t f = 0; f < n_faces; ++f) {
    if (owner[f] < 0 || owner[f] >= n_cells) return AFR_EINDEX;
    cnt[owner[f] + 1]++;
    if (!is_boundary[f] && neighbor[f] >= 0) {
      if (neighbor[f] >= n_cells) return AFR_EINDEX;
      cnt[neighbor[f] + 1]++;
    }
  }
  for (int64_t c = 0; c < n_cells; ++c) cnt[c + 1] += cnt[c];
  std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1), lst(cnt[n_cells]);
  for (int64_t f = 0; f < n_faces; ++f) {
    lst[pos[owner[f]]++] = f;
    if (!is_boundary[f] && neighbor[f] >= 0) lst[pos[neighbor[f]]++] = f;
  }
  for (int64_t f = 0; f < n_faces; ++f) colors[f] = -1;
  std::vector<uint8_t> used;
  for (int64_t f = 0; f < n_faces; ++f) {
    used.assign(used.size(), 0);
    const int64_t cells[2] = {owner[f], (!is_boundary[f] && neighbor[f] >= 0) ? neighbor[f] : -1};
    for (int64_t c : cells) {
      if (c < 0) continue;
      for (int64_t i = cnt[c]; i < cnt[c + 1]; ++i) {
        const int32_t col = colors[lst[i]];
        if (lst[i] != f && col >= 0) {
          if ((size_t)col >= used.size()) used.resize(col + 1, 0);
          used[col] = 1;
        }
      }
    }
    int32_t c = 0;
    while ((size_t)c < used.size() && used[c]) ++c;
    colors[f] = c;
  }
  return AFR_OK;
}

int afr_device_bytes(const afr_handle* h, uint64_t* out) {
  if (!h || !out) return AFR_EINVAL;
  *out = h->bytes;
  return AFR_OK;
}

int afr_destroy(afr_handle* h) {
  if (!h) return AFR_EINVAL;
  if (h->status_ev) cudaEventDestroy(h->status_ev);
  if (h->status_host) cudaFreeHost(h->status_host);
  for (void* p : h->allocs) cudaFree(p);
  delete h;
  return AFR_OK;
}

// Tables of the mixed-precision form: operator images, metric divergence,
// interior-penalty lengths, per-slot adjugate rows and the conforming-face
// match of the other side's face point.
static int mixed_setup(afr_handle* h, const afr_mesh_desc* m, const std::vector<double>* Wkeep, cudaStream_t st) {
  const int S = h->S, Fn = h->Fn, P = h->P;
  const size_t N = h->N;
  if (h->order == 3 && !h->prm.inviscid_only)
    return fail(h, AFR_EUNSUPPORTED, "the mixed form has viscous terms up to P2");
  const int Sq = pad16(S), Fq = pad16(Fn);
  int rc;
  // Conditioning: a contraction accumulated in FP32 carries an absolute error
  // of about 2^-24 * (row l1 norm of the operator) * |x|.  The collapsed-tet
  // operators grow with the order (row l1 norms ~2e4 at P1, ~2e11 at P2 and
  // ~2e8 at P3 for the reference's nodal sets), so those cell types stay in
  // the FP64 form.
  constexpr double MAX_ROW_L1 = 1e6;
  for (int t = 0; t < 2; ++t) {
    if (Wkeep[t].empty()) continue;
    auto row_l1 = [](const double* a, size_t rows, size_t cols, size_t rs, size_t cs) {
      double mx = 0.0;
      for (size_t r = 0; r < rows; ++r) {
        double acc = 0.0;
        for (size_t c = 0; c < cols; ++c) acc += std::fabs(a[r * rs + c * cs]);
        mx = std::max(mx, acc);
      }
      return mx;
    };
    double l1 = row_l1(Wkeep[t].data(), S, 3 * Fn, 3 * Fn, 1);
    l1 = std::max(l1, row_l1(m->c2f[t], Fn, S, S, 1));
    for (int mm = 0; mm < 3; ++mm) l1 = std::max(l1, row_l1(m->D_3d[t] + mm, S, S, 3 * S, 3));
    l1 = std::max(l1, row_l1(m->boundary_extrap + (size_t)t * 6 * P * S, 6 * P, S, S, 1));
    if (l1 > MAX_ROW_L1 && !h->prm.mixed_ignore_conditioning)
      return fail(h, AFR_EUNSUPPORTED,
                  std::string("the mixed form needs operators with row l1 norms <= 1e6 (FP32 accumulation); the ") +
                      (t == 0 ? "prism" : "tet") + " operators of this order reach " + std::to_string(l1));
  }
  for (int t = 0; t < 2; ++t) {
    if (Wkeep[t].empty()) continue;
    const double* c2f = m->c2f[t];
    const double* D3 = m->D_3d[t];
    const double* Wt = Wkeep[t].data();
    const double* ex = m->boundary_extrap;
    auto i_c2f = kmajor_image_cat(Fq, Sq, [&](int i, int s) { return (i < Fn && s < S) ? c2f[i * S + s] : 0.0; });
    auto i_W = kmajor_image_cat(Sq, 3 * Fq, [&](int s, int k) {
      const int mm = k / Fq, i = k % Fq;
      return (s < S && i < Fn) ? Wt[(size_t)s * 3 * Fn + i * 3 + mm] : 0.0;
    });
    auto i_D3 = kmajor_image_cat(Sq, 3 * Sq, [&](int s, int k) {
      const int mm = k / Sq, j = k % Sq;
      return (s < S && j < S) ? D3[(size_t)s * 3 * S + j * 3 + mm] : 0.0;
    });
    auto i_D3g = kmajor_image(3 * Sq, Sq, [&](int n, int j) {
      const int mm = n / Sq, s = n % Sq;
      return (s < S && j < S) ? D3[(size_t)s * 3 * S + j * 3 + mm] : 0.0;
    });
    const int edup = mx_ext_dup(6 * P);  // copies of the face-point rows (see afr_mixed.cuh)
    auto i_E = kmajor_image(128, Sq, [&](int r, int s) {
      const int fp = r % (128 / edup);
      if (fp >= 6 * P || s >= S) return 0.0;
      const int a = fp / P, i = fp % P;
      return ex[(((size_t)t * 3 + a / 2) * 2 + a % 2) * P * S + (size_t)i * S + s];
    });
    uint16_t *d_c2f, *d_W, *d_D3, *d_D3g, *d_E;
    if ((rc = upload(h, &d_c2f, i_c2f.data(), i_c2f.size(), st)) || (rc = upload(h, &d_W, i_W.data(), i_W.size(), st)) ||
        (rc = upload(h, &d_D3, i_D3.data(), i_D3.size(), st)) ||
        (rc = upload(h, &d_D3g, i_D3g.data(), i_D3g.size(), st)) || (rc = upload(h, &d_E, i_E.data(), i_E.size(), st)))
      return rc;
    if (cudaStreamSynchronize(st) != cudaSuccess) return fail(h, AFR_ECUDA, "operator image upload");
    h->mo.c2f[t] = d_c2f;
    h->mo.W[t] = d_W;
    h->mo.D3[t] = d_D3;
    h->mo.D3g[t] = d_D3g;
    h->mo.E[t] = d_E;
  }
  double *md, *hc;
  if ((rc = dalloc(h, &md, N * S * 3)) || (rc = dalloc(h, &hc, N))) return rc;
  h->mo.MD = md;
  h->mo.hcell = hc;
  float4 *adjf32, *adjs32, *invs32;
  if ((rc = dalloc(h, &adjf32, N * (size_t)h->Fn * 3)) || (rc = dalloc(h, &adjs32, N * (size_t)S * 3)) ||
      (rc = dalloc(h, &invs32, N * (size_t)S * 3)))
    return rc;
  h->mo.adjf = adjf32;
  h->mo.adjs = adjs32;
  h->mo.invs = invs32;
  double* rdet;
  if ((rc = dalloc(h, &rdet, N * (size_t)S))) return rc;
  h->mo.rdet = rdet;
  const int FW = h->order <= 2 ? 18 : 5;
  float *xf, *pfm, *jm;
  const size_t ns = h->slots.n;
  if ((rc = dalloc(h, &xf, N * FW * 6 * P)) || (rc = dalloc(h, &pfm, N * S * 20)) || (rc = dalloc(h, &jm, ns * P * 10 + 4)))  // 16 bytes of slack: the update kernel copies 16-byte-rounded slot ranges
    return rc;
  float* rv;
  if ((rc = dalloc(h, &rv, N * S * 10))) return rc;
  h->mb = MxBuf{xf, pfm, jm, rv, FW};
  float4* arow;
  uint8_t* ofp;
  if ((rc = dalloc(h, &arow, ns * P)) || (rc = dalloc(h, &ofp, ns * P))) return rc;
  h->mf = MxFace{arow, ofp};
  cudaMemsetAsync(h->status, 0, sizeof(unsigned), st);
  cudaError_t e = dispatch(h, [&](auto L) -> cudaError_t {
    using LL = decltype(L);
    const size_t nmd = N * S * 3;
    switch (h->order) {
      case 1: k_mx_md<8, 27><<<(unsigned)((nmd + 255) / 256), 256, 0, st>>>(h->g, h->ops, md);
              k_mx_hcell<8><<<(unsigned)((N + 255) / 256), 256, 0, st>>>(h->g, hc);
              if (ns) k_mx_match<8, 4><<<(unsigned)((ns * 4 + 127) / 128), 128, 0, st>>>(h->g, h->ops, h->fc, h->slots, arow, ofp, 1e-6);
              break;
      case 2: k_mx_md<27, 64><<<(unsigned)((nmd + 255) / 256), 256, 0, st>>>(h->g, h->ops, md);
              k_mx_hcell<27><<<(unsigned)((N + 255) / 256), 256, 0, st>>>(h->g, hc);
              if (ns) k_mx_match<27, 9><<<(unsigned)((ns * 9 + 127) / 128), 128, 0, st>>>(h->g, h->ops, h->fc, h->slots, arow, ofp, 1e-6);
              break;
      default: k_mx_md<64, 64><<<(unsigned)((nmd + 255) / 256), 256, 0, st>>>(h->g, h->ops, md);
              k_mx_hcell<64><<<(unsigned)((N + 255) / 256), 256, 0, st>>>(h->g, hc);
              if (ns) k_mx_match<64, 16><<<(unsigned)((ns * 16 + 127) / 128), 128, 0, st>>>(h->g, h->ops, h->fc, h->slots, arow, ofp, 1e-6);
              break;
    }
    const size_t nrows = N * (size_t)h->Fn * 3, nsrows = N * (size_t)S * 3;
    k_mx_rows_f32<<<(unsigned)((nrows + 255) / 256), 256, 0, st>>>(h->g.adj_fine, nrows, adjf32);
    k_mx_rows_f32<<<(unsigned)((nsrows + 255) / 256), 256, 0, st>>>(h->g.adj, nsrows, adjs32);
    k_mx_rows_f32<<<(unsigned)((nsrows + 255) / 256), 256, 0, st>>>(h->g.inv, nsrows, invs32);
    k_mx_rdet<<<(unsigned)((N * (size_t)S + 255) / 256), 256, 0, st>>>(h->g.det, N * (size_t)S, rdet);
    cudaError_t r = cudaGetLastError();
    return r != cudaSuccess ? r : LL::mx_grids(h);
  });
  if (e != cudaSuccess) return cuda_fail(h, e, "mixed-form set-up");
  unsigned s = 0;
  e = cudaMemcpyAsync(&s, h->status, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(h, e, "mixed-form set-up");
  cudaMemsetAsync(h->status, 0, sizeof(unsigned), st);
  // pair the matched slot points of interior faces across the face's two
  // slots: owner point (slot s, i) matched to the neighbour's face point j,
  // whose own match points back at (s's face, i)
  if (ns > 0) {
    const size_t nt = ns * P;
    std::vector<uint8_t> hofp(nt);
    std::vector<int32_t> hface(ns), hflag(ns);
    e = cudaMemcpy(hofp.data(), ofp, nt, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(hface.data(), h->slots.face, ns * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(hflag.data(), h->slots.flags, ns * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(h, e, "mixed-form face pairs");
    std::vector<int32_t> nb_slot(h->F, -1);
    for (size_t sl = 0; sl < ns; ++sl)
      if (hflag[sl] & 1) nb_slot[hface[sl]] = (int32_t)sl;
    std::vector<int2> pairs;
    std::vector<uint8_t> taken(nt, 0);
    for (size_t sl = 0; sl < ns; ++sl) {
      const int fl = hflag[sl];
      if ((fl & 1) || (fl & 2)) continue;  // owner sides of interior faces
      const int s2 = nb_slot[hface[sl]];
      if (s2 < 0) continue;
      const int code = ((fl >> 2) & 3) * 2 + ((fl & 16) ? 1 : 0);
      const int fl2 = hflag[s2];
      const int code2 = ((fl2 >> 2) & 3) * 2 + ((fl2 & 16) ? 1 : 0);
      for (int i = 0; i < P; ++i) {
        const size_t t = sl * P + i;
        const int o = hofp[t];
        if (o == MX_OFP_GENERAL || o / P != code2) continue;
        const size_t t2 = (size_t)s2 * P + o % P;
        if (hofp[t2] != code * P + i || taken[t2]) continue;
        pairs.push_back(make_int2((int)t, (int)t2));
        taken[t] = taken[t2] = 1;
      }
    }
    std::vector<int32_t> rest;
    for (size_t t = 0; t < nt; ++t)
      if (!taken[t]) rest.push_back((int32_t)t);
    int32_t* dpairs = nullptr;
    int32_t* drest = nullptr;
    if (!pairs.empty() && (rc = upload(h, &dpairs, reinterpret_cast<const int32_t*>(pairs.data()), pairs.size() * 2, st)))
      return rc;
    if (!rest.empty() && (rc = upload(h, &drest, rest.data(), rest.size(), st))) return rc;
    e = cudaStreamSynchronize(st);  // host vectors leave scope
    if (e != cudaSuccess) return cuda_fail(h, e, "mixed-form face pairs");
    h->mx_pairs = reinterpret_cast<int2*>(dpairs);
    h->mx_rest = drest;
    h->mx_npairs = (int)pairs.size();
    h->mx_nrest = (int)rest.size();
    h->mx_paired = true;
  }
  h->prec = AFR_PREC_MIXED;
  // The FP64 fine-point adjugates were needed only for MD and the FP32 copy;
  // the FP64 solution-point adjugates only for the set-up and the SST kernels.
  auto release = [&](const double*& p, size_t n) {
    auto it = std::find(h->allocs.begin(), h->allocs.end(), (void*)p);
    if (it == h->allocs.end()) return;
    h->allocs.erase(it);
    cudaFree((void*)p);
    h->bytes -= n * sizeof(double);
    p = nullptr;
  };
  release(h->g.adj_fine, N * (size_t)h->Fn * 9);
  if (h->prm.turb != AFR_TURB_SST) release(h->g.adj, N * (size_t)S * 9);
  // The dense per-record interpolation matrices are read afterwards only by
  // the general (unmatched) face points and by the SST face kernel: release
  // them when neither exists.
  if (ns && h->prm.turb != AFR_TURB_SST) {
    std::vector<uint8_t> o(ns * P);
    e = cudaMemcpy(o.data(), ofp, o.size(), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(h, e, "mixed-form set-up");
    bool all_matched = true;
    for (uint8_t v : o) all_matched = all_matched && v != MX_OFP_GENERAL;
    if (all_matched) {
      // (an indexed mesh's four pointers share one table: freed once)
      const double* mats[4] = {h->fc.nb_m0, h->fc.nb_m1, h->fc.ow_m0, h->fc.ow_m1};
      for (int i = 0; i < 4; ++i) {
        auto it = std::find(h->allocs.begin(), h->allocs.end(), (void*)mats[i]);
        if (it == h->allocs.end()) continue;
        h->allocs.erase(it);
        cudaFree((void*)mats[i]);
        h->bytes -= std::max<size_t>(h->mat_elems[i], 1) * sizeof(double);
      }
      h->fc.nb_m0 = h->fc.nb_m1 = h->fc.ow_m0 = h->fc.ow_m1 = nullptr;
    }
  }
  return AFR_OK;
}

// Order-0 tables: per-cell face references in ascending record order, the
// per-cell ghost face (the cell's last boundary face: the reference's ghost
// table holds one state per owner cell, overwritten face by face), the
// penalty code of owner-primary boundary faces and the face areas.
static int p0_setup(afr_handle* h, const afr_mesh_desc* m, cudaStream_t st) {
  const size_t N = h->N, F = h->F;
  if (F >= ((size_t)1 << 30)) return fail(h, AFR_EUNSUPPORTED, "more than 2^30 faces");
  std::vector<int32_t> ptr(N + 1, 0), last(N, -1), gface(F, -1), pen(F, 0);
  for (size_t f = 0; f < F; ++f) {
    const bool bnd = m->is_boundary[f] != 0;
    ptr[m->owner_cell[f] + 1]++;
    if (!bnd) ptr[m->neighbor_cell[f] + 1]++;
    if (bnd) last[m->owner_cell[f]] = (int32_t)f;
  }
  for (size_t c = 0; c < N; ++c) ptr[c + 1] += ptr[c];
  std::vector<int32_t> pos(ptr.begin(), ptr.end() - 1), ref(ptr[N]);
  std::vector<double> area(F);
  for (size_t f = 0; f < F; ++f) {
    const bool bnd = m->is_boundary[f] != 0;
    ref[pos[m->owner_cell[f]]++] = (int32_t)(f << 1);
    if (!bnd) ref[pos[m->neighbor_cell[f]]++] = (int32_t)((f << 1) | 1);
    if (bnd) {
      gface[f] = last[m->owner_cell[f]];
      if (m->owner_is_primary[f])
        pen[f] = 1 | ((int32_t)m->owner_axis[f] << 1) | (m->owner_side[f] > 0.0 ? 8 : 0);
    }
    area[f] = m->true_area_weight[f * (size_t)h->P];
  }
  int32_t *dptr, *dref, *dg, *dpen;
  double *dA, *flux, *fvv;
  int rc;
  if ((rc = upload(h, &dptr, ptr.data(), N + 1, st)) || (rc = upload(h, &dref, ref.data(), ref.size(), st)) ||
      (rc = upload(h, &dg, gface.data(), F, st)) || (rc = upload(h, &dpen, pen.data(), F, st)) ||
      (rc = upload(h, &dA, area.data(), F, st)) || (rc = dalloc(h, &flux, F * 8)) ||
      (rc = upload(h, &fvv, m->fv_cell_volumes ? m->fv_cell_volumes : m->cell_volumes, N, st)))
    return rc;
  if (cudaStreamSynchronize(st) != cudaSuccess) return fail(h, AFR_ECUDA, "order-0 tables");
  h->p0 = P0Tab{dptr, dref, dg, dpen, dA, fvv, flux};
  return AFR_OK;
}

int afr_create(const afr_mesh_desc* m, const afr_params* prm, void* stream, afr_handle** out) {
  if (!m || !prm || !out) return AFR_EINVAL;
  *out = nullptr;
  afr_handle* h = new afr_handle();
  auto bail = [&](int rc) {
    g_create_error = h->err;
    afr_destroy(h);
    return rc;
  };
  cudaStream_t st = (cudaStream_t)stream;
  h->N = m->n_cells;
  h->n_prism = m->n_prism;
  h->order = m->order;
  h->S = m->n_sps;
  h->Fn = m->n_fine;
  h->P = m->n_fp;
  h->F = m->n_faces;
  h->prm = *prm;
  h->nv = prm->n_vars;
  const int n1d = h->order + 1;
  if (h->order < 0 || h->order > 3) return bail(fail(h, AFR_EUNSUPPORTED, "order must be 0, 1, 2 or 3"));
  if (prm->precision != AFR_PREC_FP64 && prm->precision != AFR_PREC_MIXED)
    return bail(fail(h, AFR_EINVAL, "precision must be AFR_PREC_FP64 or AFR_PREC_MIXED"));
  if (h->order == 0 && prm->precision != AFR_PREC_FP64)
    return bail(fail(h, AFR_EUNSUPPORTED, "order 0 (finite volume) runs in the FP64 form only"));
  if (h->order == 0 && !m->true_area_weight)
    return bail(fail(h, AFR_EINVAL, "order 0 needs true_area_weight (the face areas)"));
  const int fine_1d = std::min(2 * h->order, 3) + 1;
  if (h->S != n1d * n1d * n1d || h->P != n1d * n1d || h->Fn != fine_1d * fine_1d * fine_1d)
    return bail(fail(h, AFR_EINVAL, "n_sps/n_fp/n_fine inconsistent with order"));
  if (h->nv != 5 && h->nv != 7) return bail(fail(h, AFR_EINVAL, "n_vars must be 5 or 7"));
  if (prm->turb == AFR_TURB_SST && (h->nv != 7 || !m->wall_distance))
    return bail(fail(h, AFR_EINVAL, "SST needs n_vars=7 and a wall distance field"));
  if (h->N <= 0 || h->n_prism < 0 || h->n_prism > h->N || h->F <= 0) return bail(fail(h, AFR_EINVAL, "bad sizes"));
  const size_t N = h->N, S = h->S, Fn = h->Fn, P = h->P, F = h->F;
  int rc;
  std::vector<int32_t> tmp;

  // ---- validate face tables on the host (all indices in range) ----
  for (size_t f = 0; f < F; ++f) {
    const int64_t o = m->owner_cell[f], nb = m->neighbor_cell[f];
    const bool bnd = m->is_boundary[f] != 0;
    if (o < 0 || o >= (int64_t)N || nb < -1 || nb >= (int64_t)N || (!bnd && nb < 0))
      return bail(fail(h, AFR_EINDEX, "face cell index out of range at face " + std::to_string(f)));
    if (m->owner_axis[f] < 0 || m->owner_axis[f] > 2 || (!bnd && (m->neighbor_axis[f] < 0 || m->neighbor_axis[f] > 2)))
      return bail(fail(h, AFR_EINDEX, "face axis out of range at face " + std::to_string(f)));
    for (int which = 0; which < 2; ++which) {
      const int64_t c0 = which ? m->ow_src0_cell[f] : m->nb_src0_cell[f];
      const int64_t i1 = which ? m->ow_src1_idx[f] : m->nb_src1_idx[f];
      const int64_t n1 = which ? m->n_ow_src1 : m->n_nb_src1;
      if (c0 < -1 || c0 >= (int64_t)N || i1 < -1 || i1 >= n1)
        return bail(fail(h, AFR_EINDEX, "face source index out of range at face " + std::to_string(f)));
      if (i1 >= 0) {
        const int64_t c1 = which ? m->ow_src1_cell[i1] : m->nb_src1_cell[i1];
        if (c1 < 0 || c1 >= (int64_t)N) return bail(fail(h, AFR_EINDEX, "second source cell out of range"));
      }
    }
    if (m->bc_group[f] < 0 || m->bc_group[f] >= m->n_bc) return bail(fail(h, AFR_EINDEX, "bc_group out of range"));
    if (m->colors[f] < 0) return bail(fail(h, AFR_EINVAL, "negative face color"));
  }
  for (int i = 0; i < 3 * (int)S; ++i)
    if (m->dist_fp_of_sp[i] < 0 || m->dist_fp_of_sp[i] >= (int64_t)P || m->dist_axis_coord_of_sp[i] < 0 ||
        m->dist_axis_coord_of_sp[i] >= n1d)
      return bail(fail(h, AFR_EINDEX, "distribution map out of range"));

  if ((rc = dalloc(h, &h->status, 1))) return bail(rc);
  cudaMemsetAsync(h->status, 0, sizeof(unsigned), st);
  if (cudaHostAlloc((void**)&h->status_host, sizeof(unsigned), cudaHostAllocDefault) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->status_ev, cudaEventDisableTiming) != cudaSuccess)
    return bail(fail(h, AFR_ENOMEM, "pinned status word"));
  *h->status_host = 0;

  // ---- geometry ----
  double *det = nullptr, *inv = nullptr, *detf = nullptr, *invf = nullptr;
  if ((rc = upload(h, &det, m->det_jacs, N * S, st))) return bail(rc);
  if ((rc = upload(h, &inv, m->inv_jacs, N * S * 9, st))) return bail(rc);
  double *adj, *adjf, *vol, *mfs, *wd = nullptr;
  if ((rc = dalloc(h, &adj, N * S * 9))) return bail(rc);
  if ((rc = dalloc(h, &adjf, N * Fn * 9))) return bail(rc);
  if ((rc = dalloc(h, &mfs, N * S))) return bail(rc);
  if ((rc = upload(h, &vol, m->cell_volumes, N, st))) return bail(rc);
  if (m->wall_distance && (rc = upload(h, &wd, m->wall_distance, N * S, st))) return bail(rc);
  {
    // fine-point Jacobians are only needed to form adj_fine: stage them through
    // a temporary allocation released right after
    cudaError_t e1 = cudaMalloc((void**)&detf, N * Fn * sizeof(double));
    cudaError_t e2 = cudaMalloc((void**)&invf, N * Fn * 9 * sizeof(double));
    if (e1 != cudaSuccess || e2 != cudaSuccess) {
      cudaFree(detf);
      cudaFree(invf);
      return bail(fail(h, AFR_ENOMEM, "cudaMalloc failed for fine Jacobians"));
    }
    cudaMemcpyAsync(detf, m->det_jacs_fine, N * Fn * sizeof(double), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(invf, m->inv_jacs_fine, N * Fn * 9 * sizeof(double), cudaMemcpyHostToDevice, st);
    const size_t nf = N * Fn * 9, nc = N * S * 9;
    k_form_adj<<<(unsigned)((nf + 255) / 256), 256, 0, st>>>(detf, invf, adjf, N * Fn);
    k_form_adj<<<(unsigned)((nc + 255) / 256), 256, 0, st>>>(det, inv, adj, N * S);
    if (m->metric_flux_scale)
      cudaMemcpyAsync(mfs, m->metric_flux_scale, N * S * sizeof(double), cudaMemcpyHostToDevice, st);
    else
      k_metric_flux_scale<<<(unsigned)((N * S + 255) / 256), 256, 0, st>>>(adj, mfs, N * S);
    cudaError_t e = cudaStreamSynchronize(st);
    cudaFree(detf);
    cudaFree(invf);
    if (e != cudaSuccess) return bail(cuda_fail(h, e, "geometry set-up"));
  }
  double* hvol;
  if ((rc = dalloc(h, &hvol, N))) return bail(rc);
  k_cube_root_abs<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(vol, N, hvol);
  h->g = Geom{h->N, h->n_prism, det, inv, adj, adjf, vol, mfs, wd, hvol};

  // ---- operators ----
  // fragment-major image of an M x K operator whose element (m, k) is
  // A[m * rs + k * cs] (layout in Ops)
  auto frag_image = [](const double* A, size_t M, size_t K, size_t rs, size_t cs, std::vector<double>& out) {
    const size_t MT = (M + 7) / 8, KS = (K + 3) / 4, base = out.size();
    out.resize(base + MT * KS * 32, 0.0);
    for (size_t mt = 0; mt < MT; ++mt)
      for (size_t ks = 0; ks < KS; ++ks)
        for (size_t l = 0; l < 32; ++l) {
          const size_t mm = mt * 8 + l / 4, k = ks * 4 + l % 4;
          if (mm < M && k < K) out[base + (mt * KS + ks) * 32 + l] = A[mm * rs + k * cs];
        }
  };
  auto upload_frag = [&](double** d, const double* A, size_t M, size_t K, size_t rs, size_t cs) {
    std::vector<double> img;
    frag_image(A, M, K, rs, cs, img);
    const int r = upload(h, d, img.data(), img.size(), st);
    cudaStreamSynchronize(st);  // img leaves scope
    return r;
  };
  std::vector<double> Wkeep[2];
  for (int t = 0; t < 2; ++t) {
    const bool present = t == 0 ? h->n_prism > 0 : h->N > h->n_prism;
    if (!present) continue;
    // order 0 has no over-integration operators: identity transfers and a
    // zero derivative (the finite-volume kernels do not read them)
    static const double one[1] = {1.0}, zero3[3] = {0.0, 0.0, 0.0};
    const bool p0 = h->order == 0;
    const double* c2f_h = m->c2f[t] ? m->c2f[t] : (p0 ? one : nullptr);
    const double* dfn_h = m->D_fine[t] ? m->D_fine[t] : (p0 ? zero3 : nullptr);
    const double* f2c_h = m->f2c[t] ? m->f2c[t] : (p0 ? one : nullptr);
    if (!m->D_3d[t] || !c2f_h || !dfn_h || !f2c_h || !m->filter[t])
      return bail(fail(h, AFR_EINVAL, "missing operator for a present cell type"));
    double *d3, *d3g, *c2f, *dfn, *f2c, *flt;
    if ((rc = upload(h, &d3, m->D_3d[t], S * S * 3, st))) return bail(rc);
    std::vector<double> g2(3 * S * S);
    for (size_t s = 0; s < S; ++s)
      for (int mm = 0; mm < 3; ++mm)
        for (size_t j = 0; j < S; ++j) g2[(s * 3 + mm) * S + j] = m->D_3d[t][s * 3 * S + j * 3 + mm];
    if ((rc = upload(h, &d3g, g2.data(), g2.size(), st))) return bail(rc);
    cudaStreamSynchronize(st);
    if ((rc = upload(h, &c2f, c2f_h, Fn * S, st))) return bail(rc);
    if ((rc = upload(h, &dfn, dfn_h, Fn * Fn * 3, st))) return bail(rc);
    if ((rc = upload(h, &f2c, f2c_h, S * Fn, st))) return bail(rc);
    if ((rc = upload(h, &flt, m->filter[t], S * S, st))) return bail(rc);
    // W = f2c * D_fine (S x 3Fn), summed in ascending fine-point order
    std::vector<double> Wh(S * 3 * Fn, 0.0);
    for (size_t r = 0; r < S; ++r)
      for (size_t k = 0; k < 3 * Fn; ++k) {
        double acc = 0.0;
        for (size_t i = 0; i < Fn; ++i) acc += f2c_h[r * Fn + i] * dfn_h[i * 3 * Fn + k];
        Wh[r * 3 * Fn + k] = acc;
      }
    double* wdev;
    if ((rc = upload(h, &wdev, Wh.data(), Wh.size(), st))) return bail(rc);
    cudaStreamSynchronize(st);
    h->ops.W[t] = wdev;
    {
      double *fd3, *fd3g, *fc2f, *fw, *fflt;
      if ((rc = upload_frag(&fd3, m->D_3d[t], S, 3 * S, 3 * S, 1))) return bail(rc);
      if ((rc = upload_frag(&fd3g, g2.data(), 3 * S, S, S, 1))) return bail(rc);
      if ((rc = upload_frag(&fc2f, c2f_h, Fn, S, S, 1))) return bail(rc);
      if ((rc = upload_frag(&fw, Wh.data(), S, 3 * Fn, 3 * Fn, 1))) return bail(rc);
      if ((rc = upload_frag(&fflt, m->filter[t], S, S, S, 1))) return bail(rc);
      h->ops.fD3[t] = fd3;
      h->ops.fD3g[t] = fd3g;
      h->ops.fc2f[t] = fc2f;
      h->ops.fW[t] = fw;
      h->ops.ffilt[t] = fflt;
    }
    Wkeep[t] = Wh;
    h->ops.D3[t] = d3;
    h->ops.D3g[t] = d3g;
    h->ops.c2f[t] = c2f;
    h->ops.Dfine[t] = dfn;
    h->ops.f2c[t] = f2c;
    h->ops.filt[t] = flt;
  }
  {
    double *ex, *gl, *gr;
    int32_t *dfp, *dco;
    if ((rc = upload(h, &ex, m->boundary_extrap, 12 * P * S, st))) return bail(rc);
    if ((rc = upload(h, &gl, m->g_left, (size_t)n1d, st))) return bail(rc);
    if ((rc = upload(h, &gr, m->g_right, (size_t)n1d, st))) return bail(rc);
    if ((rc = upload_i32(h, &dfp, m->dist_fp_of_sp, 3 * S, st, tmp))) return bail(rc);
    if ((rc = upload_i32(h, &dco, m->dist_axis_coord_of_sp, 3 * S, st, tmp))) return bail(rc);
    std::vector<double> fex;
    for (int q = 0; q < 12; ++q) frag_image(m->boundary_extrap + (size_t)q * P * S, P, S, S, 1, fex);
    double* fexd;
    if ((rc = upload(h, &fexd, fex.data(), fex.size(), st))) return bail(rc);
    cudaStreamSynchronize(st);  // fex leaves scope
    h->ops.fextrap = fexd;
    h->ops.extrap = ex;
    h->ops.g_left = gl;
    h->ops.g_right = gr;
    h->ops.dist_fp = dfp;
    h->ops.dist_co = dco;
  }

  // ---- faces ----
  Faces& fc = h->fc;
  fc.F = h->F;
  {
    int32_t *own, *nbr, *c0n, *i1n, *c1n, *c0o, *i1o, *c1o, *bcg;
    int8_t *oax, *nax;
    uint8_t* isb;
    double *osd, *nsd, *tn, *m0n, *m1n, *m0o, *m1o;
    if ((rc = upload_i32(h, &own, m->owner_cell, F, st, tmp))) return bail(rc);
    if ((rc = upload_i32(h, &nbr, m->neighbor_cell, F, st, tmp))) return bail(rc);
    std::vector<int8_t> ax8(F);
    for (size_t f = 0; f < F; ++f) ax8[f] = (int8_t)m->owner_axis[f];
    if ((rc = upload(h, &oax, ax8.data(), F, st))) return bail(rc);
    cudaStreamSynchronize(st);
    for (size_t f = 0; f < F; ++f) ax8[f] = (int8_t)std::max<int64_t>(m->neighbor_axis[f], 0);
    if ((rc = upload(h, &nax, ax8.data(), F, st))) return bail(rc);
    cudaStreamSynchronize(st);
    if ((rc = upload(h, &osd, m->owner_side, F, st))) return bail(rc);
    if ((rc = upload(h, &nsd, m->neighbor_side, F, st))) return bail(rc);
    if ((rc = upload(h, &isb, m->is_boundary, F, st))) return bail(rc);
    if ((rc = upload(h, &tn, m->true_normal, F * P * 3, st))) return bail(rc);
    if ((rc = upload_i32(h, &c0n, m->nb_src0_cell, F, st, tmp))) return bail(rc);
    if ((rc = upload_i32(h, &i1n, m->nb_src1_idx, F, st, tmp))) return bail(rc);
    if ((rc = upload_i32(h, &c1n, m->nb_src1_cell, (size_t)m->n_nb_src1, st, tmp))) return bail(rc);
    // interpolation matrices: an indexed mesh keeps its table of distinct
    // matrices on the device with per-record row indices; a dense mesh keeps
    // its per-record arrays with identity indices
    const bool indexed = m->src_mat_table != nullptr;
    const size_t n1n = (size_t)m->n_nb_src1, n1o = (size_t)m->n_ow_src1;
    int32_t *m0ni, *m1ni, *m0oi, *m1oi;
    if (indexed) {
      if (m->n_src_mats <= 0) return bail(fail(h, AFR_EINVAL, "empty matrix table"));
      const int32_t* idx[4] = {m->nb_src0_mat_index, m->nb_src1_mat_index, m->ow_src0_mat_index, m->ow_src1_mat_index};
      const size_t cnt[4] = {F, n1n, F, n1o};
      for (int k = 0; k < 4; ++k)
        for (size_t r = 0; r < cnt[k]; ++r)
          if (idx[k][r] < 0 || idx[k][r] >= m->n_src_mats) return bail(fail(h, AFR_EINDEX, "matrix index out of range"));
      const std::vector<double> tabT = transpose_mats(m->src_mat_table, (size_t)m->n_src_mats, P, S);
      if ((rc = upload(h, &m0n, tabT.data(), tabT.size(), st))) return bail(rc);
      cudaStreamSynchronize(st);
      m1n = m0o = m1o = m0n;
      if ((rc = upload_i32(h, &m0ni, idx[0], F, st, tmp))) return bail(rc);
      if ((rc = upload_i32(h, &m1ni, idx[1], n1n, st, tmp))) return bail(rc);
      if ((rc = upload_i32(h, &m0oi, idx[2], F, st, tmp))) return bail(rc);
      if ((rc = upload_i32(h, &m1oi, idx[3], n1o, st, tmp))) return bail(rc);
      h->mat_elems[0] = (size_t)m->n_src_mats * P * S;
    } else {
      const double* dense[4] = {m->nb_src0_mat, m->nb_src1_mat, m->ow_src0_mat, m->ow_src1_mat};
      double** dst[4] = {&m0n, &m1n, &m0o, &m1o};
      const size_t rows[4] = {F, n1n, F, n1o};
      for (int k = 0; k < 4; ++k) {
        const std::vector<double> t = transpose_mats(dense[k], rows[k], P, S);
        if ((rc = upload(h, dst[k], t.data(), t.size(), st))) return bail(rc);
        cudaStreamSynchronize(st);  // t leaves scope
      }
      std::vector<int32_t> iota(std::max<size_t>(F, std::max(n1n, n1o)));
      for (size_t r = 0; r < iota.size(); ++r) iota[r] = (int32_t)r;
      if ((rc = upload(h, &m0ni, iota.data(), F, st))) return bail(rc);
      m0oi = m0ni;
      if ((rc = upload(h, &m1ni, iota.data(), n1n, st))) return bail(rc);
      if ((rc = upload(h, &m1oi, iota.data(), n1o, st))) return bail(rc);
      cudaStreamSynchronize(st);  // iota leaves scope
      h->mat_elems[0] = F * P * S;
      h->mat_elems[1] = n1n * P * S;
      h->mat_elems[2] = F * P * S;
      h->mat_elems[3] = n1o * P * S;
    }
    if ((rc = upload_i32(h, &c0o, m->ow_src0_cell, F, st, tmp))) return bail(rc);
    if ((rc = upload_i32(h, &i1o, m->ow_src1_idx, F, st, tmp))) return bail(rc);
    if ((rc = upload_i32(h, &c1o, m->ow_src1_cell, (size_t)m->n_ow_src1, st, tmp))) return bail(rc);
    if ((rc = upload(h, &bcg, m->bc_group, F, st))) return bail(rc);
    fc.owner = own; fc.neighbor = nbr; fc.o_axis = oax; fc.n_axis = nax; fc.o_side = osd; fc.n_side = nsd;
    fc.is_bnd = isb; fc.tnormal = tn; fc.nb_c0 = c0n; fc.nb_m0 = m0n; fc.nb_i1 = i1n; fc.nb_c1 = c1n; fc.nb_m1 = m1n;
    fc.ow_c0 = c0o; fc.ow_m0 = m0o; fc.ow_i1 = i1o; fc.ow_c1 = c1o; fc.ow_m1 = m1o; fc.bc_group = bcg;
    fc.nb_m0i = m0ni; fc.nb_m1i = m1ni; fc.ow_m0i = m0oi; fc.ow_m1i = m1oi;
  }
  // slot lists: faces visited in ascending (color, face index)
  {
    std::vector<int32_t> order(F);
    for (size_t f = 0; f < F; ++f) order[f] = (int32_t)f;
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return m->colors[a] < m->colors[b]; });
    // transport slot code: face << 4 | axis << 2 | (neighbor side) << 1 | (side > 0)
    if (F >= ((size_t)1 << 27)) return bail(fail(h, AFR_EUNSUPPORTED, "more than 2^27 faces"));
    auto tcode = [&](int32_t f, bool nb) -> int32_t {
      const int ax = (int)(nb ? m->neighbor_axis[f] : m->owner_axis[f]);
      const double side = nb ? m->neighbor_side[f] : m->owner_side[f];
      return (f << 4) | (ax << 2) | (nb ? 2 : 0) | (side > 0.0 ? 1 : 0);
    };
    auto build = [&](bool transport, int32_t** dptr, int32_t** dslot) -> int {
      std::vector<int32_t> cnt(N + 1, 0);
      auto visit = [&](auto&& emit) {
        for (int32_t f : order) {
          const bool bnd = m->is_boundary[f] != 0;
          if (transport) {
            emit((int32_t)m->owner_cell[f], tcode(f, false));
            if (m->neighbor_cell[f] >= 0) emit((int32_t)m->neighbor_cell[f], tcode(f, true));
          } else {
            if (m->owner_is_primary[f]) emit((int32_t)m->owner_cell[f], f * 2);
            if (!bnd && m->neighbor_is_primary[f]) emit((int32_t)m->neighbor_cell[f], f * 2 + 1);
          }
        }
      };
      visit([&](int32_t c, int32_t) { cnt[c + 1]++; });
      for (size_t i = 0; i < N; ++i) cnt[i + 1] += cnt[i];
      std::vector<int32_t> pos(cnt.begin(), cnt.end() - 1), slots(cnt[N]);
      visit([&](int32_t c, int32_t code) { slots[pos[c]++] = code; });
      int r = upload(h, dptr, cnt.data(), N + 1, st);
      if (r) return r;
      r = upload(h, dslot, slots.data(), slots.size(), st);
      if (r) return r;
      return cudaStreamSynchronize(st) == cudaSuccess ? AFR_OK : AFR_ECUDA;
    };
    int32_t *sp, *sl, *tp, *tl;
    if ((rc = build(false, &sp, &sl))) return bail(rc);
    if ((rc = build(true, &tp, &tl))) return bail(rc);
    fc.slot_ptr = sp; fc.slot = sl; fc.tslot_ptr = tp; fc.tslot = tl;
    // slot table of the residual slots, in the same (cell, color) order
    std::vector<int32_t> ptr(N + 1), codes;
    cudaMemcpy(ptr.data(), sp, (N + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost);
    codes.resize(ptr[N]);
    cudaMemcpy(codes.data(), sl, codes.size() * sizeof(int32_t), cudaMemcpyDeviceToHost);
    const size_t ns = codes.size();
    std::vector<int32_t> sf(ns), sc(ns), sflg(ns), s0(ns), s1(ns), si1(ns);
    for (size_t c = 0; c < N; ++c)
      for (int32_t k = ptr[c]; k < ptr[c + 1]; ++k) {
        const int f = codes[k] >> 1;
        const bool nbside = (codes[k] & 1) != 0;
        const bool bnd = m->is_boundary[f] != 0;
        const int ax = (int)(nbside ? m->neighbor_axis[f] : m->owner_axis[f]);
        const double side = nbside ? m->neighbor_side[f] : m->owner_side[f];
        sf[k] = f;
        sc[k] = (int32_t)c;
        sflg[k] = (nbside ? 1 : 0) | (bnd ? 2 : 0) | (ax << 2) | (side > 0.0 ? 16 : 0);
        const int64_t i1 = nbside ? m->ow_src1_idx[f] : m->nb_src1_idx[f];
        s0[k] = bnd ? -1 : (int32_t)(nbside ? m->ow_src0_cell[f] : m->nb_src0_cell[f]);
        si1[k] = (int32_t)i1;
        s1[k] = (bnd || i1 < 0) ? -1 : (int32_t)(nbside ? m->ow_src1_cell[i1] : m->nb_src1_cell[i1]);
      }
    int32_t *d_f, *d_c, *d_fl, *d_0, *d_1, *d_i1;
    if ((rc = upload(h, &d_f, sf.data(), ns, st)) || (rc = upload(h, &d_c, sc.data(), ns, st)) ||
        (rc = upload(h, &d_fl, sflg.data(), ns, st)) || (rc = upload(h, &d_0, s0.data(), ns, st)) ||
        (rc = upload(h, &d_1, s1.data(), ns, st)) || (rc = upload(h, &d_i1, si1.data(), ns, st)))
      return bail(rc);
    cudaStreamSynchronize(st);
    h->slots = SlotTable{(int32_t)ns, d_f, d_c, d_fl, d_0, d_1, d_i1};
    // FP64 jumps: the plain stage of orders 1-3 only
    if (prm->precision != AFR_PREC_MIXED && h->order > 0 && (rc = dalloc(h, &h->J, ns * P * 10))) return bail(rc);
  }
  // ---- boundary condition table ----
  {
    int32_t *bt, *bn;
    double *bw, *bq, *bp;
    const size_t nb = (size_t)m->n_bc;
    if ((rc = upload(h, &bt, m->bc_type, nb, st))) return bail(rc);
    if ((rc = upload(h, &bn, m->bc_noslip, nb, st))) return bail(rc);
    if ((rc = upload(h, &bw, m->bc_wall_vel, nb * 3, st))) return bail(rc);
    if ((rc = upload(h, &bq, m->bc_Q, nb * 5, st))) return bail(rc);
    if ((rc = upload(h, &bp, m->bc_p_out, nb, st))) return bail(rc);
    h->bc = Bc{m->n_bc, bt, bn, bw, bq, bp};
    std::vector<uint8_t> wall(F);
    for (size_t f = 0; f < F; ++f) wall[f] = (m->is_boundary[f] && m->bc_type[m->bc_group[f]] == AFR_BC_WALL) ? 1 : 0;
    if ((rc = upload(h, &h->wall_face, wall.data(), F, st))) return bail(rc);
    cudaStreamSynchronize(st);
  }
  if (m->cd_wall_face && m->true_area_weight) {
    std::vector<int32_t> cdf;
    for (size_t f = 0; f < F; ++f)
      if (m->cd_wall_face[f] && m->owner_is_primary[f]) cdf.push_back((int32_t)f);
    h->n_cd_faces = (int)cdf.size();
    if ((rc = upload(h, &h->cd_faces, cdf.data(), cdf.size(), st))) return bail(rc);
    if ((rc = upload(h, &h->area_w, m->true_area_weight, F * P, st))) return bail(rc);
    if ((rc = dalloc(h, &h->cd_part, cdf.size() * 6))) return bail(rc);
    cudaStreamSynchronize(st);
  }
  // ---- scratch ----
  // FP64 point fields: every evaluation of the plain form; the mixed form needs
  // them only for the force integral, which allocates them for its call
  if (prm->precision != AFR_PREC_MIXED && (rc = dalloc(h, &h->PF, N * S * PFW))) return bail(rc);
  if ((rc = dalloc(h, &h->Ua, N * S * h->nv))) return bail(rc);
  if ((rc = dalloc(h, &h->Ub, N * S * h->nv))) return bail(rc);
  if ((rc = dalloc(h, &h->dt, N * S))) return bail(rc);
  if ((rc = dalloc(h, &h->norm_part, N))) return bail(rc);
  if ((rc = dalloc(h, &h->norm_rho_part, N))) return bail(rc);
  if ((rc = dalloc(h, &h->red, 4))) return bail(rc);
  if ((rc = dalloc(h, &h->red_part, (N * S + RED_CHUNK - 1) / RED_CHUNK + 1))) return bail(rc);
  if (prm->turb == AFR_TURB_SST) {
    if ((rc = dalloc(h, &h->pt, N * S * 5))) return bail(rc);
    if ((rc = dalloc(h, &h->cfp, F * P * 4))) return bail(rc);
    if ((rc = dalloc(h, &h->sp8, N * S * 8))) return bail(rc);
  }
  if (prm->precision == AFR_PREC_MIXED && (rc = mixed_setup(h, m, Wkeep, st))) return bail(rc);
  if (h->order == 0 && (rc = p0_setup(h, m, st))) return bail(rc);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return bail(cuda_fail(h, e, "afr_create"));
  *out = h;
  return AFR_OK;
}

int afr_inviscid_residual(afr_handle* h, const double* U, double* R, void* stream) {
  if (!h || !U || !R) return AFR_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  StageArgs a = base_args(h);
  a.Ucur = U;
  a.inviscid_only = 1;
  a.stage = -1;
  a.Rinv = R;
  cudaError_t e = dispatch(h, [&](auto L) { return L.eval(h, a, U, nullptr, false, st); });
  if (e != cudaSuccess) return cuda_fail(h, e, "inviscid residual");
  return check_status(h, st);
}

int afr_viscous_residual(afr_handle* h, const double* U, const double* nu_t, double* R, void* stream) {
  if (!h || !U || !R) return AFR_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  StageArgs a = base_args(h);
  a.Ucur = U;
  a.inviscid_only = 0;
  a.stage = -1;
  a.nut = nu_t;
  a.Rvisc = R;
  cudaError_t e = dispatch(h, [&](auto L) { return L.eval(h, a, U, nu_t, true, st); });
  if (e != cudaSuccess) return cuda_fail(h, e, "viscous residual");
  return check_status(h, st);
}

int afr_local_dt(afr_handle* h, const double* U, const double* nu_t, double* dt, void* stream) {
  if (!h || !U || !dt) return AFR_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  int rc = compute_dt(h, U, nu_t, dt, st);
  return rc ? rc : check_status(h, st);
}

int afr_sst_update(afr_handle* h, const double* U, const double* dt_local, double* k, double* omega, double* nu_t,
                   double* diag, void* stream) {
  if (!h || !U || !dt_local || !k || !omega || !nu_t) return AFR_EINVAL;
  if (h->prm.turb != AFR_TURB_SST) return fail(h, AFR_EINVAL, "handle was created without SST");
  cudaStream_t st = (cudaStream_t)stream;
  SstArgs s{U, dt_local, k, omega, nu_t, h->pt, h->sp8, h->cfp, h->wall_face, diag, h->nv, h->prm.mu};
  cudaError_t e = dispatch(h, [&](auto L) { return L.sst(h, s, st); });
  if (e != cudaSuccess) return cuda_fail(h, e, "sst update");
  return check_status(h, st);
}

static int step_impl(afr_handle* h, double* U, double* k, double* omega, double* nu_t, double* norm_out,
                     cudaStream_t st, StepTimer* tm, int* launches) {
  if (!h || !U) return AFR_EINVAL;
  const bool sst = h->prm.turb == AFR_TURB_SST;
  if (sst && (!k || !omega || !nu_t)) return fail(h, AFR_EINVAL, "SST step needs k, omega and nu_t");
  int rc0 = pending_status(h, st);  // a problem of an earlier step taken without a norm
  if (rc0) return rc0;
  int nl = 0;
  if (tm) tm->mark(st);
  int rc = compute_dt(h, U, sst ? nu_t : nullptr, h->dt, st);
  if (rc) return rc;
  nl += h->prm.global_dt_factor > 0.0 ? 3 : 1;
  if (tm) tm->mark(st);
  const bool visc = !h->prm.inviscid_only;
  cudaError_t e = dispatch(h, [&](auto L) {
    cudaError_t r = cudaSuccess;
    if (sst) {
      SstArgs s{U, h->dt, k, omega, nu_t, h->pt, h->sp8, h->cfp, h->wall_face, nullptr, h->nv, h->prm.mu};
      r = L.sst(h, s, st, tm);
      nl += 3;
      if (r != cudaSuccess) return r;
    }
    const double* cur[3] = {U, h->Ua, h->Ub};
    double* nxt[3] = {h->Ua, h->Ub, U};
    for (int stg = 0; stg < 3; ++stg) {
      StageArgs a = base_args(h);
      a.Ucur = cur[stg];
      a.U0 = U;
      a.Unext = nxt[stg];
      a.nut = sst ? nu_t : nullptr;
      a.dt = h->dt;
      a.norm_part = h->norm_part;
      a.norm_rho_part = h->norm_rho_part;
      a.stage = stg;
      r = L.eval(h, a, cur[stg], sst ? nu_t : nullptr, visc, st, tm, &nl);
      if (tm) tm->mark(st);
      if (r != cudaSuccess) return r;
    }
    return r;
  });
  if (e != cudaSuccess) return cuda_fail(h, e, "step");
  {
    const unsigned nb = (unsigned)(((size_t)h->N + RED_CHUNK - 1) / RED_CHUNK);
    k_reduce_chunks<false><<<nb, RED_THREADS, 0, st>>>(h->norm_part, (size_t)h->N, h->red_part);
    k_reduce_sum<<<1, 1024, 0, st>>>(h->red_part, nb, h->red);
  }
  nl += 2;
  if (tm) tm->mark(st);
  if (launches) *launches = nl;
  if (norm_out) {
    double ss = 0.0;
    e = cudaMemcpyAsync(&ss, h->red, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(h, e, "norm read");
    *norm_out = std::sqrt(ss) / std::sqrt((double)h->N * h->S * h->nv);
    return check_status(h, st);
  }
  e = queue_status_copy(h, st);
  return e == cudaSuccess ? AFR_OK : cuda_fail(h, e, "status copy");
}

int afr_step(afr_handle* h, double* U, double* k, double* omega, double* nu_t, double* norm_out, void* stream) {
  return step_impl(h, U, k, omega, nu_t, norm_out, (cudaStream_t)stream, nullptr, nullptr);
}

// ---- dual-time and IMEX integrators (core/time_integration/dual.py, imex.py) ----
namespace {
int imp_buffers(afr_handle* h) {
  if (h->iRinv) return AFR_OK;
  const size_t n = (size_t)h->N * h->S * h->nv;
  int rc;
  if ((rc = dalloc(h, &h->iRinv, n)) || (rc = dalloc(h, &h->iRvisc, n)) || (rc = dalloc(h, &h->iRscr, n)) ||
      (rc = dalloc(h, &h->iUn, n)) || (rc = dalloc(h, &h->iX, n)) || (rc = dalloc(h, &h->idt, (size_t)h->N * h->S)))
    return rc;
  return AFR_OK;
}

// inviscid and viscous residuals (dU/dt, zero turbulence columns) of the state U
int eval_both(afr_handle* h, const double* U, const double* nut, double* Rinv, double* Rvisc, cudaStream_t st) {
  StageArgs a = base_args(h);
  a.Ucur = U;
  a.inviscid_only = h->prm.inviscid_only;
  a.stage = -1;
  a.nut = nut;
  a.Rinv = Rinv;
  a.Rvisc = Rvisc;
  const bool visc = !h->prm.inviscid_only;
  cudaError_t e = dispatch(h, [&](auto L) { return L.eval(h, a, U, nut, visc, st); });
  if (e == cudaSuccess && h->prm.inviscid_only) e = cudaMemsetAsync(Rvisc, 0, (size_t)h->N * h->S * h->nv * 8, st);
  return e == cudaSuccess ? AFR_OK : cuda_fail(h, e, "residual evaluation");
}

// sqrt of the sum of squares selected by mode (see k_imp_sumsq), synchronising
int imp_norm(afr_handle* h, const ImpArgs& a, int mode, cudaStream_t st, double* out) {
  const size_t n = (size_t)a.npts * a.nv;
  const unsigned nb = (unsigned)((n + IMP_CHUNK - 1) / IMP_CHUNK);
  k_imp_sumsq<<<nb, IMP_THREADS, 0, st>>>(a, mode, h->red_part);
  k_reduce_sum<<<1, 1024, 0, st>>>(h->red_part, nb, h->red + 1);
  double ss = 0.0;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&ss, h->red + 1, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(h, e, "norm");
  *out = std::sqrt(ss);
  return AFR_OK;
}

int filter_cells(afr_handle* h, double* U, cudaStream_t st) {
  switch (h->order) {
    case 0: k_filter_cells<1><<<h->N, 32, 0, st>>>(h->g, h->ops, U, h->nv); break;
    case 1: k_filter_cells<8><<<h->N, 64, 0, st>>>(h->g, h->ops, U, h->nv); break;
    case 2: k_filter_cells<27><<<h->N, 160, 0, st>>>(h->g, h->ops, U, h->nv); break;
    default: k_filter_cells<64><<<h->N, 320, 0, st>>>(h->g, h->ops, U, h->nv); break;
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? AFR_OK : cuda_fail(h, e, "filter");
}

int copy_state(afr_handle* h, double* dst, const double* src, cudaStream_t st) {
  cudaError_t e = cudaMemcpyAsync(dst, src, (size_t)h->N * h->S * h->nv * 8, cudaMemcpyDeviceToDevice, st);
  return e == cudaSuccess ? AFR_OK : cuda_fail(h, e, "state copy");
}

// the step's preamble shared with SSP-RK3: local dt, SST once (with turb_dt),
// the residual at U^n and the RMS norm of dU/dt
int imp_preamble(afr_handle* h, double* U, double* k, double* omega, double* nu_t, const double* turb_dt,
                 double* norm_out, cudaStream_t st) {
  const bool sst = h->prm.turb == AFR_TURB_SST;
  int rc = compute_dt(h, U, sst ? nu_t : nullptr, h->dt, st);
  if (rc) return rc;
  if (sst) {
    cudaError_t e = dispatch(h, [&](auto L) {
      SstArgs s{U, turb_dt ? turb_dt : h->dt, k, omega, nu_t, h->pt, h->sp8, h->cfp, h->wall_face, nullptr, h->nv,
                h->prm.mu};
      return L.sst(h, s, st, nullptr);
    });
    if (e != cudaSuccess) return cuda_fail(h, e, "sst update");
  }
  if ((rc = eval_both(h, U, sst ? nu_t : nullptr, h->iRinv, h->iRvisc, st))) return rc;
  ImpArgs a{};
  a.npts = (int64_t)h->N * h->S;
  a.nv = h->nv;
  a.Rinv = h->iRinv;
  a.Rvisc = h->iRvisc;
  double nrm = 0.0;
  if ((rc = imp_norm(h, a, 3, st, &nrm))) return rc;
  if (norm_out) *norm_out = nrm / std::sqrt((double)h->N * h->S * h->nv);
  return AFR_OK;
}
}  // namespace

int afr_step_dual_time(afr_handle* h, double* U, double* k, double* omega, double* nu_t, double* U_prev,
                       int32_t has_prev, double dt_physical, int32_t max_inner_iter, double tol, double* norm_out,
                       void* stream) {
  if (!h || !U || !U_prev || !(dt_physical > 0.0) || max_inner_iter < 0) return AFR_EINVAL;
  const bool sst = h->prm.turb == AFR_TURB_SST;
  if (sst && (!k || !omega || !nu_t)) return fail(h, AFR_EINVAL, "SST step needs k, omega and nu_t");
  cudaStream_t st = (cudaStream_t)stream;
  if (capturing(st)) return fail(h, AFR_EINVAL, "the dual-time step synchronises: not inside a stream capture");
  int rc = pending_status(h, st);
  if (rc || (rc = imp_buffers(h))) return rc;
  const size_t npts = (size_t)h->N * h->S;
  // the SST fields advance with the physical step (core/fr_solver/step.py:109)
  k_fill_value<<<(unsigned)((npts + 255) / 256), 256, 0, st>>>(h->idt, npts, dt_physical);
  if ((rc = imp_preamble(h, U, k, omega, nu_t, h->idt, norm_out, st))) return rc;
  const double* nut = sst ? nu_t : nullptr;
  if ((rc = copy_state(h, h->iUn, U, st))) return rc;  // U^n; U itself holds the pseudo iterate
  ImpArgs a{};
  a.npts = (int64_t)npts;
  a.nv = h->nv;
  a.Rinv = h->iRinv;
  a.Rvisc = h->iRvisc;
  a.Un = h->iUn;
  a.Uprev = has_prev ? U_prev : nullptr;
  a.dtphys = dt_physical;
  a.dtl = h->dt;
  const unsigned gb = (unsigned)((npts + 255) / 256);
  double init = 0.0, prev = 0.0, cfl = 0.1;
  a.Ucur = U;
  if ((rc = imp_norm(h, a, 0, st, &init))) return rc;
  for (int it = 0; it < max_inner_iter; ++it) {
    a.Ucur = U;
    if (it > 0 && (rc = eval_both(h, U, nut, h->iRinv, h->iRvisc, st))) return rc;
    double cur = init;
    if (it > 0 && (rc = imp_norm(h, a, 0, st, &cur))) return rc;
    if (cur < init * 1e-6) break;
    if (it >= 1 && cur < tol) break;
    if (it > 0) {
      const double ratio = cur / prev;
      if (ratio < 0.5) cfl = std::min(cfl * 1.5, 10.0);
      else if (ratio > 1.0) cfl = std::max(cfl * 0.5, 0.1);
    }
    prev = cur;
    a.scale = cfl;
    // SSP-RK3 of the dual residual from U (the stage-0 residual is the one above)
    double* stg[3] = {h->Ua, h->Ub, h->iX};
    for (int s = 0; s < 3; ++s) {
      if (s > 0 && (rc = eval_both(h, stg[s - 1], nut, h->iRinv, h->iRvisc, st))) return rc;
      a.U0 = U;
      a.Ucur = s == 0 ? U : stg[s - 1];
      a.stage = s;
      a.Unext = stg[s];
      k_dual_stage<<<gb, 256, 0, st>>>(a);
      if ((rc = filter_cells(h, stg[s], st))) return rc;
    }
    // positivity and filter once more on the pseudo step's result (dual.py:137-139)
    k_positivity<<<gb, 256, 0, st>>>(h->iX, (int64_t)npts, h->nv);
    if ((rc = filter_cells(h, h->iX, st))) return rc;
    ImpArgs d = a;
    d.U0 = U;
    d.Ucur = h->iX;
    double upd = 0.0;
    if ((rc = imp_norm(h, d, 1, st, &upd))) return rc;
    if (upd < 1e-10) break;
    if ((rc = copy_state(h, U, h->iX, st))) return rc;
  }
  if ((rc = copy_state(h, U_prev, h->iUn, st))) return rc;  // level n becomes the next step's n-1
  return check_status(h, st);
}

int afr_step_imex(afr_handle* h, double* U, double* k, double* omega, double* nu_t, double* norm_out, void* stream) {
  if (!h || !U) return AFR_EINVAL;
  const bool sst = h->prm.turb == AFR_TURB_SST;
  if (sst && (!k || !omega || !nu_t)) return fail(h, AFR_EINVAL, "SST step needs k, omega and nu_t");
  cudaStream_t st = (cudaStream_t)stream;
  if (capturing(st)) return fail(h, AFR_EINVAL, "the IMEX step synchronises: not inside a stream capture");
  int rc = pending_status(h, st);
  if (rc || (rc = imp_buffers(h))) return rc;
  if ((rc = imp_preamble(h, U, k, omega, nu_t, nullptr, norm_out, st))) return rc;
  const double* nut = sst ? nu_t : nullptr;
  const size_t npts = (size_t)h->N * h->S;
  const unsigned gb = (unsigned)((npts + 255) / 256);
  // R_exp = -inviscid(U^n) stays in iRinv; iRvisc holds the viscous residual of the iterate
  ImpArgs a{};
  a.npts = (int64_t)npts;
  a.nv = h->nv;
  a.Rinv = h->iRinv;
  a.Rvisc = h->iRvisc;
  a.dtl = h->dt;
  a.Ucur = U;
  double init = 0.0, prev = 0.0, damping = 0.5;
  if ((rc = imp_norm(h, a, 2, st, &init))) return rc;
  for (int it = 0; it < 5; ++it) {
    if (it > 0 && (rc = eval_both(h, U, nut, h->iRscr, h->iRvisc, st))) return rc;
    double cur = init;
    if (it > 0 && (rc = imp_norm(h, a, 2, st, &cur))) return rc;
    if (it > 0) {
      const double ratio = cur / prev;
      if (ratio < 0.5) damping = std::min(damping * 1.2, 1.0);
      else if (ratio > 1.0) damping = std::max(damping * 0.5, 0.1);
    } else {
      damping = 0.5;
    }
    prev = cur;
    a.Ucur = U;
    a.scale = damping;
    a.Unext = h->iX;
    k_imex_update<<<gb, 256, 0, st>>>(a);
    ImpArgs d = a;
    d.U0 = U;
    d.Ucur = h->iX;
    double upd = 0.0;
    if ((rc = imp_norm(h, d, 1, st, &upd))) return rc;
    if (upd < 1e-8 || cur < init * 1e-6) break;
    if ((rc = copy_state(h, U, h->iX, st))) return rc;
  }
  return check_status(h, st);
}

// ---- launch-shape autotuner (mixed form) ----
namespace {
// device time of one residual evaluation (both residuals) with the current launch shapes, best of reps
float time_eval(afr_handle* h, const double* U, const double* nut, double* Rinv, double* Rvisc, cudaStream_t st,
                int reps) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int r = 0; r < reps + 1; ++r) {
    StageArgs a = base_args(h);
    a.Ucur = U;
    a.stage = -1;
    a.nut = nut;
    a.Rinv = Rinv;
    a.Rvisc = Rvisc;
    cudaEventRecord(e0, st);
    dispatch(h, [&](auto L) { return L.eval(h, a, U, nut, !h->prm.inviscid_only, st); });
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0) best = std::min(best, ms);  // the first run warms caches and code
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

// new[c, a, v] = sum_b W[a, b] * old[c, b, v], b ascending; one thread per output
__global__ void k_prolong(const double* __restrict__ old, int so, const double* __restrict__ W, int sn, int nc,
                          int64_t N, double* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N * sn * nc) return;
  const int v = (int)(i % nc);
  const int64_t r = i / nc;
  const int a = (int)(r % sn);
  const int64_t c = r / sn;
  const double* u = old + c * so * nc + v;
  const double* w = W + (size_t)a * so;
  double acc = 0.0;
  for (int b = 0; b < so; ++b) acc += w[b] * u[(size_t)b * nc];
  out[i] = acc;
}

__global__ void k_segment_sums(const double* __restrict__ part, const int64_t* __restrict__ ptr, double* out) {
  __shared__ double sh[256];
  double acc = 0.0;
  for (int64_t i = ptr[blockIdx.x] + threadIdx.x; i < ptr[blockIdx.x + 1]; i += blockDim.x) acc += part[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}
}  // namespace

int afr_autotune(afr_handle* h, const double* U, const double* nu_t, int32_t* choice_out, void* stream) {
  if (!h || !U) return AFR_EINVAL;
  if (h->prec != AFR_PREC_MIXED) {
    if (choice_out) choice_out[0] = choice_out[1] = choice_out[2] = -1;
    return AFR_OK;  // the plain form keeps its fixed shapes
  }
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n = (size_t)h->N * h->S * h->nv;
  double *Ri = nullptr, *Rv = nullptr;
  if (cudaMalloc((void**)&Ri, n * sizeof(double)) != cudaSuccess || cudaMalloc((void**)&Rv, n * sizeof(double)) != cudaSuccess) {
    cudaFree(Ri);
    return fail(h, AFR_ENOMEM, "autotune scratch");
  }
  const double* nut = h->prm.turb == AFR_TURB_SST ? nu_t : nullptr;
  // coordinate search: pre-pass CTAs per SM, face-kernel block, update-kernel cells per CTA
  {
    int best = h->mx_pre_per_sm;
    float tb = 1e30f;
    for (int c = 1; c <= h->mx_pre_max_per_sm; ++c) {
      h->mx_pre_per_sm = c;
      h->mx_pre_blocks = c * h->n_sms;
      const float t = time_eval(h, U, nut, Ri, Rv, st, 3);
      if (t < tb) { tb = t; best = c; }
    }
    h->mx_pre_per_sm = best;
    h->mx_pre_blocks = best * h->n_sms;
  }
  {
    const int cand[3] = {64, 128, 256};
    int best = h->mx_face_block;
    float tb = 1e30f;
    for (int c : cand) {
      h->mx_face_block = c;
      const float t = time_eval(h, U, nut, Ri, Rv, st, 3);
      if (t < tb) { tb = t; best = c; }
    }
    h->mx_face_block = best;
  }
  {
    int best = h->mx_upd_var;
    float tb = 1e30f;
    for (int c = 0; c < 3; ++c) {
      h->mx_upd_var = c;
      const float t = time_eval(h, U, nut, Ri, Rv, st, 3);
      if (t < tb) { tb = t; best = c; }
    }
    h->mx_upd_var = best;
  }
  cudaError_t e = cudaStreamSynchronize(st);
  cudaFree(Ri);
  cudaFree(Rv);
  if (e != cudaSuccess) return cuda_fail(h, e, "autotune");
  if (choice_out) {
    choice_out[0] = h->mx_pre_per_sm;
    choice_out[1] = h->mx_face_block;
    choice_out[2] = h->mx_upd_var;
  }
  return check_status(h, st);
}

int afr_launch_shape(const afr_handle* h, int32_t* out) {
  if (!h || !out) return AFR_EINVAL;
  const bool mx = h->prec == AFR_PREC_MIXED;
  const int32_t v[8] = {mx ? h->mx_pre_per_sm : -1, mx ? h->mx_pre_max_per_sm : -1, mx ? h->mx_pre_occ : -1,
                        mx && h->n_sms ? h->mx_cell_blocks / h->n_sms : -1, mx ? h->mx_vol_occ : -1,
                        mx ? h->mx_face_block : -1, mx ? h->mx_upd_var : -1, h->n_sms};
  for (int i = 0; i < 8; ++i) out[i] = v[i];
  return AFR_OK;
}

int afr_segment_norms(afr_handle* h, int32_t nseg, const int64_t* cell_ptr, int32_t which, double* out,
                      void* stream) {
  if (!h || nseg <= 0 || !cell_ptr || !out || (which != 0 && which != 1)) return AFR_EINVAL;
  if (cell_ptr[0] < 0 || cell_ptr[nseg] > h->N) return fail(h, AFR_EINVAL, "segment bounds outside the mesh");
  for (int i = 0; i < nseg; ++i)
    if (cell_ptr[i + 1] < cell_ptr[i]) return fail(h, AFR_EINVAL, "segment pointers must not decrease");
  cudaStream_t st = (cudaStream_t)stream;
  int64_t* dptr = nullptr;
  double* dsum = nullptr;
  if (cudaMalloc((void**)&dptr, (nseg + 1) * sizeof(int64_t)) != cudaSuccess ||
      cudaMalloc((void**)&dsum, nseg * sizeof(double)) != cudaSuccess) {
    cudaFree(dptr);
    return fail(h, AFR_ENOMEM, "segment scratch");
  }
  std::vector<double> sums(nseg);
  cudaMemcpyAsync(dptr, cell_ptr, (nseg + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st);
  k_segment_sums<<<nseg, 256, 0, st>>>(which ? h->norm_rho_part : h->norm_part, dptr, dsum);
  cudaMemcpyAsync(sums.data(), dsum, nseg * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  cudaFree(dptr);
  cudaFree(dsum);
  if (e != cudaSuccess) return cuda_fail(h, e, "segment norms");
  for (int i = 0; i < nseg; ++i) {
    const double cnt = (double)(cell_ptr[i + 1] - cell_ptr[i]) * h->S * (which ? 1 : h->nv);
    out[i] = cnt > 0 ? std::sqrt(sums[i]) / std::sqrt(cnt) : 0.0;
  }
  return AFR_OK;
}

int afr_residual_sums(afr_handle* h, double* out2, void* stream) {
  if (!h || !out2) return AFR_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  const unsigned nb = (unsigned)(((size_t)h->N + RED_CHUNK - 1) / RED_CHUNK);
  // the same fixed-order two-level sums as the step norm, into the handle's
  // reduction scratch, then both results to the caller's device buffer
  k_reduce_chunks<false><<<nb, RED_THREADS, 0, st>>>(h->norm_part, (size_t)h->N, h->red_part);
  k_reduce_sum<<<1, 1024, 0, st>>>(h->red_part, nb, h->red + 2);
  k_reduce_chunks<false><<<nb, RED_THREADS, 0, st>>>(h->norm_rho_part, (size_t)h->N, h->red_part);
  k_reduce_sum<<<1, 1024, 0, st>>>(h->red_part, nb, h->red + 3);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out2, h->red + 2, 2 * sizeof(double), cudaMemcpyDeviceToDevice, st);
  return e == cudaSuccess ? AFR_OK : cuda_fail(h, e, "residual sums");
}

int afr_status(afr_handle* h, int32_t nseg, const int64_t* cell_ptr, int32_t* seg_status, int32_t clear,
               void* stream) {
  if (!h || nseg < 0 || (nseg > 0 && (!cell_ptr || !seg_status))) return AFR_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  if (capturing(st)) return fail(h, AFR_EINVAL, "afr_status synchronises: not inside a stream capture");
  unsigned s = 0;
  cudaError_t e = cudaMemcpyAsync(&s, h->status, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(h, e, "status read");
  if (nseg > 0) {
    // a segment whose stage-0 norm partials of the last step are not all
    // finite holds a non-finite value; partials are sums of squares, so their
    // per-segment sum is finite exactly when every partial is
    std::vector<double> sums(nseg);
    int rc = afr_segment_norms(h, nseg, cell_ptr, 0, sums.data(), stream);
    if (rc) return rc;
    for (int i = 0; i < nseg; ++i) seg_status[i] = std::isfinite(sums[i]) ? AFR_OK : AFR_ENONFINITE;
  }
  const int code = status_code(h, s);
  if (clear) {
    e = cudaMemsetAsync(h->status, 0, sizeof(unsigned), st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(h, e, "status clear");
    *h->status_host = 0;
  }
  h->status_pending = false;
  return code;
}

int afr_step_profile(afr_handle* h, double* U, double* k, double* omega, double* nu_t, double* ms_out, int n_ms,
                     int* launches, void* stream) {
  if (!h || !ms_out || n_ms < 1) return AFR_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  StepTimer tm;
  for (int i = 0; i < 24; ++i) cudaEventCreate(&tm.ev[i]);
  int rc = step_impl(h, U, k, omega, nu_t, nullptr, st, &tm, launches);
  if (rc == AFR_OK) {
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = cuda_fail(h, e, "profile sync");
  }
  for (int i = 0; i < n_ms; ++i) ms_out[i] = -1.0;
  if (rc == AFR_OK)
    for (int i = 0; i + 1 < tm.n && i < n_ms; ++i) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, tm.ev[i], tm.ev[i + 1]);
      ms_out[i] = ms;
    }
  for (int i = 0; i < 24; ++i) cudaEventDestroy(tm.ev[i]);
  return rc;
}

int afr_prolong(afr_handle* h, const double* old_field, int32_t n_sps_old, int32_t n_cols, const double* W,
                double* new_field, void* stream) {
  if (!h || !old_field || !W || !new_field) return AFR_EINVAL;
  if (n_sps_old < 1 || n_sps_old > 64 || n_cols < 1 || n_cols > 8)
    return fail(h, AFR_EINVAL, "prolong: n_sps_old must be 1..64 and n_cols 1..8");
  const size_t n_old = (size_t)h->N * n_sps_old * n_cols, n_new = (size_t)h->N * h->S * n_cols;
  const uintptr_t o = reinterpret_cast<uintptr_t>(old_field), nw = reinterpret_cast<uintptr_t>(new_field);
  if (o < nw + n_new * sizeof(double) && nw < o + n_old * sizeof(double))
    return fail(h, AFR_EINVAL, "prolong: old and new fields overlap");
  int rc;
  if (!h->wprol && (rc = dalloc(h, &h->wprol, 64 * 64))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(h->wprol, W, (size_t)h->S * n_sps_old * sizeof(double), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_fail(h, e, "prolong matrix");
  if (n_new > 0)
    k_prolong<<<(unsigned)((n_new + 255) / 256), 256, 0, st>>>(old_field, n_sps_old, h->wprol, h->S, n_cols,
                                                                (int64_t)h->N, new_field);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(h, e, "prolong");
  // W may be pageable memory the caller frees on return: finish the copy
  e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? AFR_OK : cuda_fail(h, e, "prolong");
}

int afr_cd_cl(afr_handle* h, const double* U, const double* nu_t, double reference_area, double* out3, void* stream) {
  if (!h || !U || !out3) return AFR_EINVAL;
  if (!h->cd_faces) return fail(h, AFR_EINVAL, "handle was created without wall-face force tables");
  cudaStream_t st = (cudaStream_t)stream;
  // mixed handles keep no FP64 point fields between calls: a temporary set here
  double* pf_tmp = nullptr;
  if (!h->PF) {
    if (cudaMalloc((void**)&pf_tmp, (size_t)h->N * h->S * PFW * sizeof(double)) != cudaSuccess)
      return fail(h, AFR_ENOMEM, "force: point fields");
    h->PF = pf_tmp;
  }
  cudaError_t e = dispatch(h, [&](auto L) {
    cudaError_t r = L.pre(h, U, nu_t, true, st);
    return r != cudaSuccess ? r : L.force(h, U, nu_t, st);
  });
  if (pf_tmp) {
    cudaError_t e2 = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = e2;
    cudaFree(pf_tmp);
    h->PF = nullptr;
  }
  if (e != cudaSuccess) return cuda_fail(h, e, "force");
  std::vector<double> part((size_t)h->n_cd_faces * 6);
  e = cudaMemcpyAsync(part.data(), h->cd_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(h, e, "force read");
  double Fp[3] = {0, 0, 0}, Fv[3] = {0, 0, 0};
  for (int i = 0; i < h->n_cd_faces; ++i)
    for (int d = 0; d < 3; ++d) {
      Fp[d] += part[i * 6 + d];
      Fv[d] += -part[i * 6 + 3 + d];
    }
  const double q = 0.5 * h->prm.rho_inf * h->prm.vel_inf * h->prm.vel_inf;
  const double den = std::max(q * reference_area, 1e-300);
  out3[0] = (Fp[0] + Fv[0]) / den;
  out3[1] = (Fp[2] + Fv[2]) / den;
  out3[2] = (Fp[1] + Fv[1]) / den;
  return AFR_OK;
}

}  // extern "C"
