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
  double* norm_rho_part;  // (N) per-cell sum of squares of the density column of dU/dt (stage 0)
  int nv;
  int stage;            // 0,1,2 RK stage, -1 residual only
  int inviscid_only;
  double mu;
  unsigned* status;
  int N;                     // cells
  const int32_t* slot_flags; // (n_slots) flags of the residual slots (see SlotTable)
  int cell_base, cell_end;   // cell range of this launch (one cell type)
};

__device__ __forceinline__ int cell_type(const Geom& g, int e) { return e < g.n_prism ? 0 : 1; }

// Doubles per point of a state tile staged in shared memory (n_vars <= 7 used).
// Odd, so that threads reading consecutive points' rows hit different banks.
constexpr int US = 9;

// asynchronous 8-byte copy global -> shared (both 8-byte aligned); completed
// by cp_async_wait_all before the block barrier that publishes the data
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
// 16-byte asynchronous copy global -> shared (both 16-byte aligned)
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// one m8n8k4 FP64 step: lane (g = lane/4, t = lane%4) supplies A[g][t] and
// B[t][g] and holds D[g][2t], D[g][2t+1]
__device__ __forceinline__ void dmma884(double& d0, double& d1, double a0, double b0) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a0), "d"(b0));
}


// Small FP64 products C (M x N) = A (M x K) * B (K x N) on the FP64 tensor
// path: mma.sync m8n8k4 .f64, one 8 x 8 output tile per warp at a time, K in
// steps of 4.  A is read from a fragment-major image (layout in Ops): one
// contiguous 256-byte load per warp and k-step, the image's zeros standing for
// the rows and columns outside the operator; b(k, n) fetches B (padding reads
// as zero) and c(m, n, value) stores results; block-wide work split by warp,
// no barrier inside.  The sum order over k is the unit's, so results can
// differ from a sequential FP64 sum in the last bits.
template <class FB, class FC>
__device__ __forceinline__ void dmma_product_f(int M, int N, int K, const double* __restrict__ Af, FB b, FC c) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int nw = blockDim.x >> 5;
  const int mt = (M + 7) >> 3, nt = (N + 7) >> 3, KS = (K + 3) >> 2;
  for (int tile = threadIdx.x >> 5; tile < mt * nt; tile += nw) {
    const int mi = tile / nt, m = mi * 8 + g, n0 = (tile % nt) * 8;
    const double* ap = Af + (size_t)mi * KS * 32 + lane;
    double c0 = 0.0, c1 = 0.0;
    for (int ks = 0; ks < KS; ++ks) {
      const int k = ks * 4 + t;
      const double a0 = __ldg(ap + ks * 32);
      const double b0 = (k < K && n0 + g < N) ? b(k, n0 + g) : 0.0;
      dmma884(c0, c1, a0, b0);
    }
    const int n = n0 + 2 * t;
    if (m < M) {
      if (n < N) c(m, n, c0);
      if (n + 1 < N) c(m, n + 1, c1);
    }
  }
}

// dmma_product_f with each warp computing all column tiles of a row tile
// (at most NT of them): the A fragment is loaded once per k-step and the NT
// accumulations are independent, so their tensor-core latencies overlap.  Per
// element the k-steps accumulate in the same order as dmma_product_f.  Pays
// when the row tiles keep every warp busy (measured: slower than
// dmma_product_f for the 27-row filter and SST divergence with 4 row tiles).
template <int NT, class FB, class FC>
__device__ __forceinline__ void dmma_product_rb(int M, int N, int K, const double* __restrict__ Af, FB b, FC c) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int nw = blockDim.x >> 5;
  const int mt = (M + 7) >> 3, KS = (K + 3) >> 2;
  for (int mi = threadIdx.x >> 5; mi < mt; mi += nw) {
    const double* ap = Af + (size_t)mi * KS * 32 + lane;
    double acc[NT][2];
#pragma unroll
    for (int ni = 0; ni < NT; ++ni) acc[ni][0] = acc[ni][1] = 0.0;
    for (int ks = 0; ks < KS; ++ks) {
      const int k = ks * 4 + t;
      const double a0 = __ldg(ap + ks * 32);
#pragma unroll
      for (int ni = 0; ni < NT; ++ni) {
        const int n = ni * 8 + g;
        const double b0 = (k < K && n < N) ? b(k, n) : 0.0;
        dmma884(acc[ni][0], acc[ni][1], a0, b0);
      }
    }
    const int m = mi * 8 + g;
    if (m < M) {
#pragma unroll
      for (int ni = 0; ni < NT; ++ni) {
        const int n = ni * 8 + 2 * t;
        if (n < N) c(m, n, acc[ni][0]);
        if (n + 1 < N) c(m, n + 1, acc[ni][1]);
      }
    }
  }
}

// Median-based outlier zeroing (core/fr_operators/troubled_cell.py:346-408):
// per cell and variable, |R| > 1e4 * max(median |R|, 1e-9 mean|U|, 1e-300)
// is set to zero.  A column has nothing to zero when that threshold is at
// least max |R|.  Two lower bounds of the median prove that without ranking:
// the minimum, and p = max|R| * 1e-4 (raised until 1e4 * p >= max|R|) when at
// least as many elements as lie at or above the median's rank are >= p.
// Such columns (no NaN) skip the O(S^2) rank pass; the others take it, so the
// result is the same element for element.
constexpr int OUT_WORK = 25;  // [0,5) median or bound, [5,10) mean|U|, [10,20) middle pair, [20,25) rank flag

// per column v of one block: mean |U| (rows Ur, stride ldU), the bound and the rank flag
template <int S>
__device__ __forceinline__ void outlier_column(const double* R, const double* Ur, int ldU, int v, double* w) {
  constexpr int NEED = S - ((S & 1) ? S / 2 : S / 2 - 1);  // elements at or above the (lower) middle rank
  double acc = 0.0, lo = INFINITY, hi = 0.0;
  bool nan = false;
  for (int s = 0; s < S; ++s) {
    acc += fabs(Ur[s * ldU + v]);
    const double x = fabs(R[s * 5 + v]);
    lo = fmin(lo, x);
    hi = fmax(hi, x);
    nan = nan || isnan(x);
  }
  w[5 + v] = acc / S;
  const double fl = 1e-9 * w[5 + v];
  bool skip = !nan && hi <= 1e4 * fmax(fmax(lo, fl), 1e-300);
  double bound = lo;
  if (!nan && !skip) {
    double p = hi * 1e-4;
    // next double up (p is finite and >= 0 here: its bit pattern plus one)
    for (int it = 0; it < 4 && 1e4 * p < hi; ++it) p = __longlong_as_double(__double_as_longlong(p) + 1);
    if (1e4 * p >= hi) {
      int cnt = 0;
      for (int s = 0; s < S; ++s) cnt += fabs(R[s * 5 + v]) >= p;
      if (cnt >= NEED) {
        skip = true;
        bound = p;
      }
    }
  }
  w[v] = bound;
  w[20 + v] = skip ? 0.0 : 1.0;
}

// stable rank of |R[s,v]| in its column; the middle one(s) into w
template <int S>
__device__ __forceinline__ void outlier_rank(const double* R, int s, int v, double* w) {
  const double x = fabs(R[s * 5 + v]);
  int rank = 0;
  for (int j = 0; j < S; ++j) {
    const double y = fabs(R[j * 5 + v]);
    rank += (y < x) || (y == x && j < s);
  }
  if (S & 1) {
    if (rank == S / 2) w[v] = x;
  } else {
    if (rank == S / 2 - 1) w[10 + v] = x;
    if (rank == S / 2) w[15 + v] = x;
  }
}

__device__ __forceinline__ void outlier_zero(double* R, int r, int v, const double* w, bool odd) {
  const double med = odd ? w[v] : 0.5 * (w[10 + v] + w[15 + v]);
  const double ref = fmax(fmax(med, 1e-9 * w[5 + v]), 1e-300);
  if (fabs(R[r]) > 1e4 * ref) R[r] = 0.0;
}

// nb contiguous (S,5) blocks R + b*S*5 in shared memory, reference rows
// Uref + b*S*ldU (first 5 columns), all blocks in one pass per phase.  work >= OUT_WORK doubles per block.
template <int S>
__device__ void suppress_outliers_blocks(double* R, const double* Uref, int ldU, int nb, double* work) {
  int flagged = 0;
  for (int t = threadIdx.x; t < nb * 5; t += blockDim.x) {
    const int b = t / 5, v = t % 5;
    outlier_column<S>(R + b * S * 5, Uref + b * S * ldU, ldU, v, work + b * OUT_WORK);
    flagged |= work[b * OUT_WORK + 20 + v] != 0.0;
  }
  if (!__syncthreads_or(flagged)) return;  // no column takes the rank pass: nothing is zeroed
  for (int t = threadIdx.x; t < nb * S * 5; t += blockDim.x) {
    const int b = t / (S * 5), r = t % (S * 5), s = r / 5, v = r % 5;
    double* w = work + b * OUT_WORK;
    if (w[20 + v] != 0.0) outlier_rank<S>(R + b * S * 5, s, v, w);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nb * S * 5; t += blockDim.x) {
    const int b = t / (S * 5), r = t % (S * 5), v = r % 5;
    const double* w = work + b * OUT_WORK;
    if (w[20 + v] != 0.0) outlier_zero(R + b * S * 5, r, v, w, S & 1);
  }
  __syncthreads();
}

// The same for the inviscid and viscous residuals of nc cells at once: block
// b < nc is sRi of cell b, block nc + b is sRv of cell b; cell rows of the
// reference field at sU + b*S*US.  work >= OUT_WORK doubles per block.
template <int S>
__device__ void suppress_outliers_cells(double* sRi, double* sRv, const double* sU, int nc, bool visc, double* work) {
  const int nb = nc * (visc ? 2 : 1);
  int flagged = 0;
  for (int t = threadIdx.x; t < nb * 5; t += blockDim.x) {
    const int bb = t / 5, v = t % 5;
    const double* R = bb < nc ? sRi + bb * S * 5 : sRv + (bb - nc) * S * 5;
    outlier_column<S>(R, sU + (bb % nc) * S * US, US, v, work + bb * OUT_WORK);
    flagged |= work[bb * OUT_WORK + 20 + v] != 0.0;
  }
  if (!__syncthreads_or(flagged)) return;  // no column takes the rank pass: nothing is zeroed
  for (int t = threadIdx.x; t < nb * S * 5; t += blockDim.x) {
    const int bb = t / (S * 5), r = t % (S * 5), s = r / 5, v = r % 5;
    double* w = work + bb * OUT_WORK;
    if (w[20 + v] != 0.0) outlier_rank<S>(bb < nc ? sRi + bb * S * 5 : sRv + (bb - nc) * S * 5, s, v, w);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nb * S * 5; t += blockDim.x) {
    const int bb = t / (S * 5), r = t % (S * 5), v = r % 5;
    const double* w = work + bb * OUT_WORK;
    if (w[20 + v] != 0.0) outlier_zero(bb < nc ? sRi + bb * S * 5 : sRv + (bb - nc) * S * 5, r, v, w, S & 1);
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
struct PreTile {
  static constexpr int CPB = S <= 8 ? 16 : (S <= 27 ? 4 : 2);  // cells per CTA
};

// CPB cells per CTA; cells [cell_base, cell_end) share one cell type.  The
// reference-space gradients are one FP64 tensor-core product (rows s*3+m of
// D3g, columns (cell, field)); the tile's PF rows are assembled in shared
// memory and stored as one contiguous block.
template <int S>
__global__ void __launch_bounds__(128) k_pre(Geom g, Ops ops, const double* __restrict__ U, int nv,
                                             const double* __restrict__ nut, int want_grads,
                                             double* __restrict__ PF, int cell_base, int cell_end) {
  constexpr int CPB = PreTile<S>::CPB;
  __shared__ double sPF[CPB * S * PFW];
  __shared__ double f[CPB * S * 4];
  __shared__ double gc[CPB * S * 3 * 4];
  const int e0 = cell_base + blockIdx.x * CPB;
  const int nc = min(CPB, cell_end - e0);
  const int ct = cell_type(g, e0);
  for (int t = threadIdx.x; t < nc * S; t += blockDim.x) {
    const size_t p = (size_t)e0 * S + t;
    double q[5];
    const double* u = U + p * nv;
    cons_to_prim(u, q);
    double* o = sPF + t * PFW;
    for (int v = 0; v < 5; ++v) o[v] = q[v];
    o[17] = nut ? fmax(u[0], 1e-10) * nut[p] : 0.0;
    f[t * 4 + 0] = q[1];
    f[t * 4 + 1] = q[2];
    f[t * 4 + 2] = q[3];
    f[t * 4 + 3] = q[4] / (fmax(q[0], 1e-10) * R_AIR);
  }
  __syncthreads();
  if (want_grads) {
    dmma_product_rb<(4 * CPB + 7) / 8>(
        3 * S, 4 * nc, S, ops.fD3g[ct], [&](int j, int col) { return f[((col >> 2) * S + j) * 4 + (col & 3)]; },
        [&](int r, int col, double x) { gc[((col >> 2) * S * 3 + r) * 4 + (col & 3)] = x; });
    __syncthreads();
    for (int t = threadIdx.x; t < nc * S; t += blockDim.x) {
      double inv[9];
      const double* ip = g.inv + ((size_t)e0 * S + t) * 9;
      for (int k = 0; k < 9; ++k) inv[k] = __ldg(ip + k);
      for (int c = 0; c < 12; ++c) {
        const int q = c / 3, n = c % 3;  // c = q*3+n: q in (u,v,w,T)
        double acc = 0.0;
        for (int m = 0; m < 3; ++m) acc += gc[(t * 3 + m) * 4 + q] * inv[m * 3 + n];
        sPF[t * PFW + 5 + c] = acc;
      }
    }
  } else {
    for (int t = threadIdx.x; t < nc * S * 12; t += blockDim.x) sPF[(t / 12) * PFW + 5 + t % 12] = 0.0;
  }
  __syncthreads();
  double* out = PF + (size_t)e0 * S * PFW;
  for (int t = threadIdx.x; t < nc * S * PFW; t += blockDim.x) out[t] = sPF[t];
}

// ---------------------------------------------------------------------------
// face kernel: one thread per (slot, flux point).  A slot is one side of one
// face record whose own extrapolation + correction lifting lands on a cell
// (core/fr_residual/inviscid_kernel_colored.py:86-157 owner side, :159-236
// neighbour side; core/fr_residual/viscous_flux_kernel.py:335-520).  Writes
// the inviscid and viscous flux jumps J (n_slots, NP, 10).
// Slot flags: bit0 neighbour side, bit1 boundary face, bits2-3 axis, bit4 side>0.
// ---------------------------------------------------------------------------
struct SlotTable {
  int32_t n;                // number of slots
  const int32_t* face;      // (n)
  const int32_t* cell;      // (n) cell the slot lifts into
  const int32_t* flags;     // (n)
  const int32_t* c0;        // (n) first interpolation source cell, -1 if none
  const int32_t* c1;        // (n) second source cell, -1 if none
  const int32_t* i1;        // (n) row of the compact second-source table
};



// one warp's m8n8k4 FP64 product C (M x N) = A (M x K) * B (K x N) with
// every tile's accumulators held in registers (MT row tiles, NT column
// tiles): each k-step loads the A fragments of all row tiles and the B
// fragments of all column tiles, so the operand loads of the whole product
// are independent of one another and of the products.  a(m, k), b(k, n)
// fetch operands (padding reads as zero), c(m, n, value) stores results.
template <int MT, int NT, int K, class FA, class FB, class FC>
__device__ __forceinline__ void dmma_warp_rb(int M, int N, FA a, FB b, FC c) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  double acc[MT][NT][2];
#pragma unroll
  for (int mi = 0; mi < MT; ++mi)
#pragma unroll
    for (int ni = 0; ni < NT; ++ni) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;
#pragma unroll
  for (int k0 = 0; k0 < K; k0 += 4) {
    const int k = k0 + t;
    double av[MT], bv[NT];
#pragma unroll
    for (int mi = 0; mi < MT; ++mi) {
      const int m = mi * 8 + g;
      av[mi] = (m < M && k < K) ? a(m, k) : 0.0;
    }
#pragma unroll
    for (int ni = 0; ni < NT; ++ni) {
      const int n = ni * 8 + g;
      bv[ni] = (n < N && k < K) ? b(k, n) : 0.0;
    }
#pragma unroll
    for (int mi = 0; mi < MT; ++mi)
#pragma unroll
      for (int ni = 0; ni < NT; ++ni) dmma884(acc[mi][ni][0], acc[mi][ni][1], av[mi], bv[ni]);
  }
#pragma unroll
  for (int mi = 0; mi < MT; ++mi)
#pragma unroll
    for (int ni = 0; ni < NT; ++ni) {
      const int m = mi * 8 + g, n = ni * 8 + 2 * t;
      if (m < M) {
        if (n < N) c(m, n, acc[mi][ni][0]);
        if (n + 1 < N) c(m, n + 1, acc[mi][ni][1]);
      }
    }
}

// dmma_warp_rb with A read from a fragment-major image (layout in Ops) of an
// operator with at most MT * 8 rows and K columns
template <int MT, int NT, int K, class FB, class FC>
__device__ __forceinline__ void dmma_warp_rb_f(int M, int N, const double* __restrict__ Af, FB b, FC c) {
  constexpr int KS = (K + 3) / 4;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  double acc[MT][NT][2];
#pragma unroll
  for (int mi = 0; mi < MT; ++mi)
#pragma unroll
    for (int ni = 0; ni < NT; ++ni) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;
#pragma unroll
  for (int ks = 0; ks < KS; ++ks) {
    const int k = ks * 4 + t;
    double av[MT], bv[NT];
#pragma unroll
    for (int mi = 0; mi < MT; ++mi) av[mi] = __ldg(Af + (mi * KS + ks) * 32 + lane);
#pragma unroll
    for (int ni = 0; ni < NT; ++ni) {
      const int n = ni * 8 + g;
      bv[ni] = (n < N && k < K) ? b(k, n) : 0.0;
    }
#pragma unroll
    for (int mi = 0; mi < MT; ++mi)
#pragma unroll
      for (int ni = 0; ni < NT; ++ni) dmma884(acc[mi][ni][0], acc[mi][ni][1], av[mi], bv[ni]);
  }
#pragma unroll
  for (int mi = 0; mi < MT; ++mi)
#pragma unroll
    for (int ni = 0; ni < NT; ++ni) {
      const int m = mi * 8 + g, n = ni * 8 + 2 * t;
      if (m < M) {
        if (n < N) c(m, n, acc[mi][ni][0]);
        if (n + 1 < N) c(m, n + 1, acc[mi][ni][1]);
      }
    }
}

// Face kernel: one warp per group of SPW = 32 / NP slots (a slot is one side
// of one face record whose correction lifts into a cell; lane = slot-in-group
// * NP + flux point in the flux phase).  Per slot, the own side's
// extrapolation E * [q, adjugate row of the face's axis, grads, mu_t] and the
// other side's interpolation M_src0 * [q, grads, mu_t] (+ M_src1 * ...) are
// FP64 tensor-core products into the warp's shared rows; the lanes then form
// the ghost state, AUSM+up with the alignment fallback and the BR1 common
// flux with the boundary penalty
// (core/fr_residual/inviscid_kernel_colored.py:86-236,
// core/fr_residual/viscous_flux_kernel.py:335-520) and write the jumps
// J (n_slots, NP, 10).  A weight of zero contributes nothing to the products
// while the state is finite (the reference skips zero weights,
// inviscid_kernel_colored.py:117-121; a non-finite state makes the step
// non-finite either way).
// Slot flags: bit0 neighbour side, bit1 boundary face, bits2-3 axis, bit4 side>0.
constexpr int FACE_WARPS = 4;
constexpr int FW_OWN = 21, FW_OTH = 18;  // doubles per face point: own side, other side

template <int S, int NP>
__global__ void __launch_bounds__(32 * FACE_WARPS, 4) k_face(Geom g, Ops ops, Faces fc, Bc bc, SlotTable st,
                                                          const double* __restrict__ PF, double mu, int visc,
                                                          double* __restrict__ J) {
  constexpr int SPW = 32 / NP;  // slots per warp
  constexpr int MT = (NP + 7) / 8;  // row tiles of the face points
  __shared__ double sOw[FACE_WARPS][SPW * NP * FW_OWN];
  __shared__ double sOt[FACE_WARPS][SPW * NP * FW_OTH];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sl0 = (blockIdx.x * FACE_WARPS + warp) * SPW;
  if (sl0 >= st.n) return;  // whole warps leave together
  const int nsl = min(SPW, st.n - sl0);
  double* ow_s = sOw[warp];
  double* ot_s = sOt[warp];
  for (int j = 0; j < nsl; ++j) {
    const int sl = sl0 + j;
    const int f = st.face[sl];
    const int e = st.cell[sl];
    const int fl = st.flags[sl];
    const bool is_owner = (fl & 1) == 0;
    const bool bnd = (fl & 2) != 0;
    const int ax = (fl >> 2) & 3;
    const int sb = (fl & 16) ? 1 : 0;
    const int ct = cell_type(g, e);
    // own side: rows face points, columns [q(5), adj row(3), grads + mu_t(13)]
    const double* Ef = ops.fextrap + (((size_t)ct * 3 + ax) * 2 + sb) * (MT * ((S + 3) / 4) * 32);
    const double* pf = PF + (size_t)e * S * PFW;
    const double* ad = g.adj + (size_t)e * S * 9 + ax * 3;
    double* ow = ow_s + j * NP * FW_OWN;
    {
      auto fb = [&](int s, int n) {
        return n < 5 ? __ldg(pf + s * PFW + n) : (n < 8 ? __ldg(ad + s * 9 + (n - 5)) : __ldg(pf + s * PFW + n - 3));
      };
      auto fc_ = [&](int i, int n, double x) { ow[i * FW_OWN + n] = x; };
      if (visc) dmma_warp_rb_f<MT, 3, S>(NP, FW_OWN, Ef, fb, fc_);
      else dmma_warp_rb_f<MT, 1, S>(NP, 8, Ef, fb, fc_);  // columns 8.. are not read without viscosity
    }
    // other side: the interpolation sources (the first, then the second added)
    double* ot = ot_s + j * NP * FW_OTH;
    if (!bnd) {
      for (int src = 0; src < 2; ++src) {
        const int c = src == 0 ? st.c0[sl] : st.c1[sl];
        if (c < 0) {
          if (src == 0)
            for (int t = lane; t < NP * FW_OTH; t += 32) ot[t] = 0.0;
          continue;
        }
        const double* M = src == 0 ? (is_owner ? fmat(fc.nb_m0, fc.nb_m0i, f, 0, NP, S)
                                               : fmat(fc.ow_m0, fc.ow_m0i, f, 0, NP, S))
                                   : (is_owner ? fmat(fc.nb_m1, fc.nb_m1i, st.i1[sl], 0, NP, S)
                                               : fmat(fc.ow_m1, fc.ow_m1i, st.i1[sl], 0, NP, S));
        const double* pc = PF + (size_t)c * S * PFW;
        __syncwarp();
        auto fa = [&](int i, int s) { return __ldg(M + s * NP + i); };
        auto fb = [&](int s, int n) { return __ldg(pc + s * PFW + n); };
        auto fc_ = [&](int i, int n, double x) {
          if (src == 0) ot[i * FW_OTH + n] = x;
          else ot[i * FW_OTH + n] += x;
        };
        if (visc) dmma_warp_rb<MT, 3, S>(NP, FW_OTH, fa, fb, fc_);
        else dmma_warp_rb<MT, 1, S>(NP, 5, fa, fb, fc_);  // columns 5.. are not read without viscosity
      }
    }
  }
  __syncwarp();
  // flux phase: lane = slot-in-group * NP + face point
  const int j = lane / NP, i = lane % NP;
  if (j >= nsl || lane >= SPW * NP) return;
  const int sl = sl0 + j;
  const int f = st.face[sl];
  const int e = st.cell[sl];
  const int fl = st.flags[sl];
  const bool is_owner = (fl & 1) == 0;
  const bool bnd = (fl & 2) != 0;
  const double side = (fl & 16) ? 1.0 : -1.0;
  double ow[21], ot[18];
#pragma unroll
  for (int k = 0; k < 21; ++k) ow[k] = (k < 8 || visc) ? ow_s[(j * NP + i) * FW_OWN + k] : 0.0;
  const double* tn = fc.tnormal + ((size_t)f * NP + i) * 3;
  if (bnd) {
    double qo[5], n[3], gq[5];
    for (int v = 0; v < 5; ++v) qo[v] = ow[v];
    for (int d = 0; d < 3; ++d) n[d] = tn[d];
    ghost_state(bc, fc.bc_group[f], qo, n, gq);
    for (int v = 0; v < 5; ++v) ot[v] = gq[v];
    for (int k = 0; k < 13; ++k) ot[5 + k] = ow[8 + k];
  } else {
#pragma unroll
    for (int k = 0; k < 18; ++k) ot[k] = (k < 5 || visc) ? ot_s[(j * NP + i) * FW_OTH + k] : 0.0;
  }
  // pointwise fluxes
  const double a0 = ow[5], a1 = ow[6], a2 = ow[7];
  double mag = sqrt(a0 * a0 + a1 * a1 + a2 * a2);
  if (mag < 1e-300) mag = 1e-300;
  double dir[3] = {a0 / mag * side, a1 / mag * side, a2 / mag * side};
  const double sg = is_owner ? 1.0 : -1.0;
  const double t0 = sg * tn[0], t1 = sg * tn[1], t2 = sg * tn[2];
  if (dir[0] * t0 + dir[1] * t1 + dir[2] * t2 < 0.5) { dir[0] = t0; dir[1] = t1; dir[2] = t2; }
  double Fc[5], Fp[3][5];
  ausm_up(ow, ot, dir, Fc);
  euler_flux(ow, Fp);
  double* Jo = J + ((size_t)sl * NP + i) * 10;
  for (int v = 0; v < 5; ++v) Jo[v] = Fc[v] * mag * side - (a0 * Fp[0][v] + a1 * Fp[1][v] + a2 * Fp[2][v]);
  if (visc) {
    double qa[5], ga[13];
    for (int v = 0; v < 5; ++v) qa[v] = 0.5 * (ow[v] + ot[v]);
    for (int k = 0; k < 13; ++k) ga[k] = 0.5 * (ow[8 + k] + ot[5 + k]);
    double Gc[3][5], Go[3][5];
    viscous_flux(qa, ga, ga + 9, mu, ga[12], Gc);
    viscous_flux(ow, ow + 8, ow + 17, mu, ow[20], Go);
    double jv[5];
    for (int v = 0; v < 5; ++v)
      jv[v] = (a0 * Gc[0][v] + a1 * Gc[1][v] + a2 * Gc[2][v]) - (a0 * Go[0][v] + a1 * Go[1][v] + a2 * Go[2][v]);
    if (bnd) {
      // interior-penalty term on boundary faces (core/fr_operators/flux_kernels.py:140-200);
      // cell volume scale = mean of det over the cell's points (viscous_flux_kernel.py:344-347)
      double vol_o = 0.0;
      for (int s = 0; s < S; ++s) vol_o += g.det[(size_t)e * S + s];
      vol_o /= S;
      double h = pow(vol_o, 1.0 / 3.0);
      if (h < 1e-300) h = 1e-300;
      const double eta = C_IP * (mu + ow[20]) / h;
      const double scale = eta * sqrt(a0 * a0 + a1 * a1 + a2 * a2) * side;
      for (int v = 1; v < 4; ++v) jv[v] += -scale * (ow[v] - ot[v]);
    }
    for (int v = 0; v < 5; ++v) Jo[5 + v] = jv[v];
  }
}

// ---------------------------------------------------------------------------
// cell kernel: CPB cells per CTA.  Volume terms (inviscid over-integrated
// divergence with W = f2c * D_fine folded at create, viscous divergence),
// lifting of the face jumps of each cell's slots in ascending color order,
// outlier suppression, then (stage >= 0) the SSP-RK3 Shu-Osher combination,
// positivity projection and modal filter (core/time_integration/base.py:250-335,
// core/time_integration/positivity.py:13-45, core/fr_solver/filter.py:29-42).
// ---------------------------------------------------------------------------
constexpr int CELL_THREADS = 256;
constexpr int CELL_MAXSLOT = 6;  // slots per cell staged in shared memory (more: read from global)

template <int S, int FN, int CPB, int NPMAX>
struct CellSmem {
  static constexpr int oPF = 0;                    // CPB*S*18
  static constexpr int oAdj = oPF + CPB * S * PFW; // CPB*S*9
  static constexpr int oU = oAdj + CPB * S * 9;    // CPB*S*US
  static constexpr int oDet = oU + CPB * S * US;    // CPB*S
  static constexpr int oRi = oDet + CPB * S;       // CPB*S*5
  static constexpr int oRv = oRi + CPB * S * 5;    // CPB*S*5
  static constexpr int oQf = oRv + CPB * S * 5;    // CPB*FN*5
  static constexpr int oFt = oQf + CPB * FN * 5;   // CPB*FN*15
  static constexpr int oGt = oFt + CPB * FN * 15;  // CPB*S*15
  static constexpr int oJ = oGt + CPB * S * 15;    // staged jumps of the CTA's slots
  static constexpr int oWp = oJ + CPB * CELL_MAXSLOT * NPMAX * 10;  // 2 halves of the W divergence
  static constexpr int oAf = oWp + 2 * CPB * S * 5;  // CPB*FN*9 adjugates at the fine points
  static constexpr int work = oAf + CPB * FN * 9;     // CPB*2*OUT_WORK (outliers) + 32
  static constexpr int total = work + CPB * 2 * OUT_WORK + 32;
};

template <int S, int FN, int NP, int CPB>
__global__ void __launch_bounds__(CELL_THREADS, 3) k_cell(Geom g, Ops ops, Faces fc, StageArgs a,
                                                          const double* __restrict__ J) {
  using L = CellSmem<S, FN, CPB, NP>;
  extern __shared__ double sm[];
  double* sPF = sm + L::oPF;
  double* sAdj = sm + L::oAdj;
  double* sU = sm + L::oU;
  double* sDet = sm + L::oDet;
  double* sRi = sm + L::oRi;
  double* sRv = sm + L::oRv;
  double* sQf = sm + L::oQf;
  double* sFt = sm + L::oFt;
  double* sGt = sm + L::oGt;
  double* work = sm + L::work;
  const int e0 = a.cell_base + blockIdx.x * CPB;
  const int nc = min(CPB, a.cell_end - e0);
  const int ct = cell_type(g, e0);  // a launch covers cells of one type
  const int nv = a.nv;
  const bool visc = !a.inviscid_only;
  const int tid = threadIdx.x;

  double* sAf = sm + L::oAf;
  // ---- load: asynchronous 8-byte copies, all in flight at once ----
  for (int t = tid; t < nc * S * PFW; t += blockDim.x) cp_async8(sPF + t, a.PF + (size_t)e0 * S * PFW + t);
  for (int t = tid; t < nc * S * 9; t += blockDim.x) cp_async8(sAdj + t, g.adj + (size_t)e0 * S * 9 + t);
  for (int t = tid; t < nc * S * nv; t += blockDim.x)
    cp_async8(sU + (t / nv) * US + t % nv, a.Ucur + (size_t)e0 * S * nv + t);
  for (int t = tid; t < nc * S; t += blockDim.x) cp_async8(sDet + t, g.det + (size_t)e0 * S + t);
  for (int t = tid; t < nc * FN * 9; t += blockDim.x) cp_async8(sAf + t, g.adj_fine + (size_t)e0 * FN * 9 + t);
  // the jumps of this CTA's slots are contiguous (slots are stored cell-major)
  const int k_beg = fc.slot_ptr[e0], k_end = fc.slot_ptr[e0 + nc];
  const bool staged = (k_end - k_beg) <= CPB * CELL_MAXSLOT;
  double* sJ = sm + L::oJ;
  if (staged)
    for (int t = tid; t < (k_end - k_beg) * NP * 10; t += blockDim.x)
      cp_async8(sJ + t, J + (size_t)k_beg * NP * 10 + t);
  cp_async_wait_all();
  __syncthreads();

  // ---- Q at fine points (c2f, an FP64 tensor-core product: rows the fine
  // points, columns (cell, variable)) and viscous contravariant fluxes ----
  {
    dmma_product_rb<(5 * CPB + 7) / 8>(
        FN, 5 * nc, S, ops.fc2f[ct],
        [&](int s, int col) { return sPF[((col / 5) * S + s) * PFW + col % 5]; },
        [&](int i, int col, double x) { sQf[((col / 5) * FN + i) * 5 + col % 5] = x; });
  }
  if (visc) {
    for (int t = tid; t < nc * S; t += blockDim.x) {
      double q[5], G[3][5];
      const double* p = sPF + t * PFW;
      for (int v = 0; v < 5; ++v) q[v] = p[v];
      viscous_flux(q, p + 5, p + 14, a.mu, p[17], G);
      const double* am = sAdj + t * 9;
      for (int m = 0; m < 3; ++m)
        for (int v = 0; v < 5; ++v)
          sGt[(t * 3 + m) * 5 + v] = am[m * 3 + 0] * G[0][v] + am[m * 3 + 1] * G[1][v] + am[m * 3 + 2] * G[2][v];
    }
  }
  __syncthreads();
  // ---- Euler fluxes at fine points, contravariant with adj_fine ----
  for (int t = tid; t < nc * FN; t += blockDim.x) {
    const int b = t / FN, i = t % FN;
    double q[5], F[3][5];
    for (int v = 0; v < 5; ++v) q[v] = sQf[t * 5 + v];
    euler_flux(q, F);
    const double* ad = sAf + (size_t)(b * FN + i) * 9;
    double am[9];
    for (int k = 0; k < 9; ++k) am[k] = ad[k];
    for (int m = 0; m < 3; ++m)
      for (int v = 0; v < 5; ++v)
        sFt[(t * 3 + m) * 5 + v] = am[m * 3 + 0] * F[0][v] + am[m * 3 + 1] * F[1][v] + am[m * 3 + 2] * F[2][v];
  }
  __syncthreads();
  // ---- divergences on the FP64 tensor path: inviscid W (S x 3FN) applied to
  // the fine-point fluxes, viscous D3 (S x 3S) to the point fluxes; rows the
  // solution points, columns (cell, variable) ----
  {
    dmma_product_f(
        S, 5 * nc, FN * 3, ops.fW[ct],
        [&](int k, int col) { return sFt[(col / 5) * FN * 15 + k * 5 + col % 5]; },
        [&](int s, int col, double x) {
          const int b = col / 5;
          sRi[(b * S + s) * 5 + col % 5] = -x / sDet[b * S + s];
        });
    if (visc) {
      dmma_product_f(
          S, 5 * nc, S * 3, ops.fD3[ct],
          [&](int k, int col) { return sGt[(col / 5) * S * 15 + k * 5 + col % 5]; },
          [&](int s, int col, double x) {
            const int b = col / 5;
            sRv[(b * S + s) * 5 + col % 5] = x / sDet[b * S + s];
          });
    }
  }
  __syncthreads();
  // ---- lift the face jumps of each cell's slots, ascending color order ----
  for (int t = tid; t < nc * S * 5; t += blockDim.x) {
    const int b = t / (S * 5), r = t % (S * 5), s = r / 5, v = r % 5;
    const int e = e0 + b;
    const double rdj = 1.0 / sDet[b * S + s];  // each term within an ulp of g' J / det
    double ci = 0.0, cv = 0.0;
    for (int k = fc.slot_ptr[e]; k < fc.slot_ptr[e + 1]; ++k) {
      const int fl = a.slot_flags[k];
      const int ax = (fl >> 2) & 3;
      const int fp = ops.dist_fp[ax * S + s];
      const double gw = ((fl & 16) ? ops.g_right : ops.g_left)[ops.dist_co[ax * S + s]];
      const double* Jk = staged ? sJ + ((k - k_beg) * NP + fp) * 10 : J + ((size_t)k * NP + fp) * 10;
      ci += -(gw * Jk[v]) * rdj;
      if (visc) cv += (gw * Jk[5 + v]) * rdj;
    }
    sRi[t] = sRi[t] + ci;
    if (visc) sRv[t] = sRv[t] + cv;
  }
  __syncthreads();
  suppress_outliers_cells<S>(sRi, sRv, sU, nc, visc, work);

  if (a.stage < 0) {
    for (int t = tid; t < nc * S * nv; t += blockDim.x) {
      const int p = t / nv, v = t % nv;
      if (a.Rinv) a.Rinv[(size_t)e0 * S * nv + t] = v < 5 ? sRi[p * 5 + v] : 0.0;
      if (a.Rvisc) a.Rvisc[(size_t)e0 * S * nv + t] = (v < 5 && visc) ? sRv[p * 5 + v] : 0.0;
    }
    return;
  }

  // ---- RK stage combination + positivity (per point) ----
  double* Up = sQf;  // (CPB*S, US) reuses the fine-point scratch (and the flux scratch after it)
  static_assert(CPB * S * US <= CPB * FN * 20, "RK tile must fit the fine-point and flux scratch");
  double* part = sGt;  // (CPB*S) squared dU/dt per point (stage 0)
  // loops over the 8 possible variables, unrolled, so the arrays stay in registers
  for (int p = tid; p < nc * S; p += blockDim.x) {
    double Lr[8], un[8];
    double sq_sum = 0.0;
#pragma unroll
    for (int v = 0; v < 8; ++v) Lr[v] = v < 5 ? sRi[p * 5 + v] + (visc ? sRv[p * 5 + v] : 0.0) : 0.0;
#pragma unroll
    for (int v = 0; v < 8; ++v)
      if (v < nv) sq_sum += Lr[v] * Lr[v];
    const size_t gp = (size_t)e0 * S + p;
    const double dts = a.dt[gp];
    const double* u0 = a.U0 + gp * nv;
    const double* uc = sU + p * US;
    if (a.stage == 0) {
#pragma unroll
      for (int v = 0; v < 8; ++v) un[v] = v < nv ? u0[v] + dts * Lr[v] : 0.0;
    } else if (a.stage == 1) {
#pragma unroll
      for (int v = 0; v < 8; ++v) un[v] = v < nv ? (0.75 * u0[v] + 0.25 * uc[v]) + (0.25 * dts) * Lr[v] : 0.0;
    } else {
      // 1/3 U0 + 0 U1 + 2/3 U2 + 2/3 dt L; the 0*U1 term is dropped: it can only
      // turn a finite value into NaN where U1 is non-finite, and U2 (filtered
      // from U1) is then non-finite at the same cell already.
#pragma unroll
      for (int v = 0; v < 8; ++v)
        un[v] = v < nv ? (1.0 / 3.0 * u0[v] + 2.0 / 3.0 * uc[v]) + (2.0 / 3.0 * dts) * Lr[v] : 0.0;
    }
    const double rho = fmax(un[0], 1e-6);
    un[0] = rho;
    double vel[3] = {un[1] / rho, un[2] / rho, un[3] / rho};
    const double vm = sqrt(vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
    if (vm > 1e4) {
      const double cf = 1e4 / vm;
      for (int d = 0; d < 3; ++d) { vel[d] *= cf; un[1 + d] = rho * vel[d]; }
    }
    const double ke = 0.5 * rho * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
    const double pr = (GAMMA - 1.0) * (un[4] - ke);
    if (pr < 1.0) un[4] = 1.0 / (GAMMA - 1.0) + ke;
    if (nv > 5) un[5] = fmax(un[5], 0.0);
    if (nv > 6) un[6] = fmax(un[6], 1e-8);
#pragma unroll
    for (int v = 0; v < 8; ++v)
      if (v < nv) Up[p * US + v] = un[v];
    part[p] = sq_sum;
    part[CPB * S + p] = Lr[0] * Lr[0];
  }
  __syncthreads();
  // modal filter on the first five variables as an FP64 tensor-core product
  // (rows s, columns (cell, variable), K the cell's points)
  dmma_product_f(
      S, 5 * nc, S, ops.ffilt[ct],
      [&](int j, int col) { return Up[((col / 5) * S + j) * US + col % 5]; },
      [&](int s, int col, double x) { a.Unext[((size_t)(e0 + col / 5) * S + s) * nv + col % 5] = x; });
  for (int p = tid; p < nc * S; p += blockDim.x)
    for (int v = 5; v < nv; ++v) a.Unext[((size_t)e0 * S + p) * nv + v] = Up[p * US + v];
  if (a.stage == 0 && tid < nc) {
    double acc = 0.0;  // fixed order per cell: points ascending
    for (int s = 0; s < S; ++s) acc += part[tid * S + s];
    a.norm_part[e0 + tid] = acc;
    double acc_rho = 0.0;
    for (int s = 0; s < S; ++s) acc_rho += part[CPB * S + tid * S + s];
    a.norm_rho_part[e0 + tid] = acc_rho;
    // a non-finite dU/dt anywhere in the cell makes its partial non-finite
    if (!isfinite(acc) && a.status) atomicOr(a.status, (unsigned)DS_NONFINITE);
  }
}

}  // namespace afr
