// Mixed-precision form of the FR residual-and-update stage.
//
// The operator contractions run on the tensor cores (tcgen05, BF16 inputs,
// FP32 accumulation in tensor memory) as three-term hi+lo split products,
// D = A_hi*B_hi + A_hi*B_lo + A_lo*B_hi, which carry about 16 significant bits
// of each factor.  Pointwise fluxes are FP32.  FP64 is kept for the state, the
// geometry metrics, the primitive recovery from the conserved state, the
// residual sums and RK update, the norm and the force coefficients.
//
// Four kernels per stage (same data flow as the reference's residual,
// core/fr_residual/inviscid.py:139-345 and core/fr_residual/viscous_flux.py:113-302):
//   k_mx_pre   per 8-cell tile: gradients of (u,v,w,T) (D_3d as a GEMM) and the
//              extrapolation of all point fields to every face point of the
//              cell (boundary_extrap of all six faces stacked as one GEMM);
//   k_mx_face  per (slot, flux point): AUSM+up and BR1 jumps.  Where the
//              other side's interpolation row equals one of that cell's own
//              extrapolation rows (matched once at create: every prism face
//              point, most tet face points) the other side is read from its
//              face-point fields; elsewhere it is interpolated from the source
//              cells' FP32 point fields with the reference's matrices;
//   k_mx_vol   per C-cell tile (persistent): c2f, viscous D_3d and the folded
//              W = f2c*D_fine divergence as GEMMs -> volume terms (FP32);
//   k_mx_update per few cells: lifting in ascending color order, outlier
//              zeroing, SSP-RK3 combination, positivity (FP64), filter (an
//              FP64 product on the tensor path).
//
// Contraction inputs are deviations from the cell mean where the operator
// reproduces constants (c2f, extrapolation, derivatives), so the split error is
// relative to the variation inside the cell, not to the free-stream level.  The
// inviscid flux is split as F(q) = F(qbar) + dF: the W contraction acts on the
// contravariant dF (formed algebraically, without cancellation), and
// W*(adj_fine (x) F(qbar)) = MD*F(qbar) uses the FP64 metric divergence
// MD[c,s,n] = sum_{i,m} W[s,(i,m)] adj_fine[c,i,m,n] formed at create.
//
// Shared-memory operand images are K-major without swizzle (afr_tc.cuh).  Row
// orders are chosen so that lanes of a warp write eight consecutive 16-byte
// rows (conflict-free 2-byte stores): A rows are (field, cell) with the cell
// index fastest in groups of eight.
#pragma once
#include "afr_kernels.cuh"
#include "afr_tc.cuh"

namespace afr {

constexpr int MX_THREADS = 512;  // pre-pass CTA
constexpr int MX_PRE_CELLS = 8;

__host__ __device__ constexpr int pad16(int x) { return (x + 15) / 16 * 16; }
__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }
__host__ __device__ constexpr int pow2_cols(int x) { return x <= 32 ? 32 : (x <= 64 ? 64 : (x <= 128 ? 128 : 256)); }
// Copies of the face-point rows in the 128-row extrapolation image: with 6*NP
// face points <= 32 (P1) every 32-lane quarter of tensor memory holds a copy,
// <= 64 (P2) two halves do; each copy's readout serves its share of the tile's
// cells, so every warp of the CTA takes part in the readout.
__host__ __device__ constexpr int mx_ext_dup(int nfp) { return nfp <= 32 ? 4 : (nfp <= 64 ? 2 : 1); }

// Operator images, K-major canonical, BF16 bit patterns.  "cat" images stack
// the hi rows over the lo rows (2N rows, one image); the others are [hi | lo].
struct MxOps {
  const uint16_t* c2f[2];  // B cat: rows i < Fq (fine point), K = Sq (solution point)
  const uint16_t* W[2];    // B cat: rows s < Sq, K = 3*Fq, k = m*Fq + i
  const uint16_t* D3[2];   // B cat: rows s < Sq, K = 3*Sq, k = m*Sq + j
  const uint16_t* D3g[2];  // B: rows m*Sq + s, K = Sq (j)
  const uint16_t* E[2];    // A: rows j*(128/DUP) + fp, fp = (ax*2+side)*NP + i, copies j < DUP = mx_ext_dup(6*NP); K = Sq
  const double* MD;        // (N, S, 3) metric divergence of the folded W
  const float4* adjf;      // (N, FN, 3) FP32 fine-point adjugate rows (4th entry zero)
  const float4* adjs;      // (N, S, 3) FP32 solution-point adjugate rows
  const float4* invs;      // (N, S, 3) FP32 inverse-Jacobian rows
  const double* rdet;      // (N, S) 1 / det, FP64
  const double* hcell;     // (N) interior-penalty length, cube root of the mean det
};

constexpr uint8_t MX_OFP_GENERAL = 255;  // other side by interpolation from point fields

struct MxFace {
  const float4* arow;   // (n_slots*NP) own adjugate row at the flux point, and its norm
  const uint8_t* ofp;   // (n_slots*NP) face point of the other side, (ax*2+side)*NP + j, or MX_OFP_GENERAL
};

struct MxBuf {
  float* XF;   // (N, FW, 6*NP) point fields at every face point of the cell
  float* PFm;  // (N, S, 20) gradients of u, v, w, T (12), mu_t, q (5), 2 unused
  float* Jm;   // (n_slots, NP, 10) inviscid and viscous jumps
  float* RV;   // (N, S, 10) inviscid and viscous volume terms
  int FW;      // 18 (q 5, grads 12, mu_t) or 5 (inviscid handles)
};

namespace mxd {

__device__ __forceinline__ void st_split(uint16_t* img, int img_elems, int idx, float x) {
  const __nv_bfloat16 h = __float2bfloat16_rn(x);
  const __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
  img[idx] = __bfloat16_as_ushort(h);
  img[img_elems + idx] = __bfloat16_as_ushort(l);
}

// n floats, 16-byte vector accesses when both ends allow them
__device__ __forceinline__ void copy_f32(float* dst, const float* src, int n) {
  if (((reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src)) & 15u) == 0) {
    const float4* s4 = reinterpret_cast<const float4*>(src);
    float4* d4 = reinterpret_cast<float4*>(dst);
    for (int t = threadIdx.x; t < n / 4; t += blockDim.x) d4[t] = s4[t];
    for (int t = (n / 4) * 4 + threadIdx.x; t < n; t += blockDim.x) dst[t] = src[t];
  } else {
    for (int t = threadIdx.x; t < n; t += blockDim.x) dst[t] = src[t];
  }
}

// L2 prefetch of bytes [off, off + bytes) of an array of total bytes (bulk
// copy engine, no data returned to the SM); the range is clipped to 16-byte
// boundaries inside the array.  A hint: issued by one thread.
__device__ __forceinline__ void prefetch_l2(const void* base, size_t total, size_t off, size_t bytes) {
  const size_t lo = off & ~size_t(15);
  size_t hi = off + bytes;
  hi = (hi + 15) & ~size_t(15);
  const size_t cap = total & ~size_t(15);
  if (hi > cap) hi = cap;
  const uintptr_t b = reinterpret_cast<uintptr_t>(base);
  for (size_t p = lo; p < hi; p += 32768) {
    const uint32_t n = (uint32_t)((hi - p) < 32768 ? (hi - p) : 32768);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(b + p), "r"(n) : "memory");
  }
}

// two consecutive K positions (idx even) of one row: hi and lo parts as
// packed bf16x2 words, one conversion per part
__device__ __forceinline__ void st_split2(uint16_t* img, int img_elems, int idx, float x0, float x1) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
  *reinterpret_cast<__nv_bfloat162*>(img + idx) = h;
  *reinterpret_cast<__nv_bfloat162*>(img + img_elems + idx) = l;
}

// (cell, point pair) enumeration with the cell fastest in groups of 8: lanes
// of a warp cover 8 cells x 4 consecutive pairs (8 points, one 16-byte row each)
__device__ __forceinline__ void cell_pair(int idx, int npts, int& c, int& p0) {
  const int rest = idx >> 3;
  p0 = 2 * (rest % (npts / 2));
  c = (rest / (npts / 2)) * 8 + (idx & 7);
}

using afr::cp_async8;
using afr::cp_async_wait_all;

// 16-byte copy global -> shared of an operator image
__device__ __forceinline__ void copy_img(void* dst, const void* src, int bytes) {
  const uint4* s = reinterpret_cast<const uint4*>(src);
  uint4* d = reinterpret_cast<uint4*>(dst);
  for (int t = threadIdx.x; t < bytes / 16; t += blockDim.x) d[t] = __ldg(s + t);
}

// D (tensor memory) = A * B^T over K with the three-term split; A has 128
// rows, B has nb rows.  Issued by one thread.
__device__ __forceinline__ void mma_split(uint32_t tmem, const uint16_t* A, const uint16_t* B, int nb, int K) {
  const uint32_t a_hi = tc::smem_u32(A), a_lo = a_hi + 128u * K * 2u;
  const uint32_t b_hi = tc::smem_u32(B), b_lo = b_hi + (uint32_t)nb * K * 2u;
  const uint32_t idesc = tc::idesc_bf16(128, nb);
  for (int ks = 0; ks < K / 16; ++ks) {
    const uint32_t ao = ks * 2u * 128u * 16u, bo = ks * 2u * (uint32_t)nb * 16u;
    const uint64_t ah = tc::make_desc(a_hi + ao, 128 * 16, 128), al = tc::make_desc(a_lo + ao, 128 * 16, 128);
    const uint64_t bh = tc::make_desc(b_hi + bo, nb * 16, 128), bl = tc::make_desc(b_lo + bo, nb * 16, 128);
    tc::mma_bf16(tmem, ah, bh, idesc, ks > 0 ? 1u : 0u);
    tc::mma_bf16(tmem, ah, bl, idesc, 1u);
    tc::mma_bf16(tmem, al, bh, idesc, 1u);
  }
}

// D (tensor memory, 2n columns) with the three-term split against a stacked
// operator image Bcat = [B_hi; B_lo] (2n rows): columns [0, n) collect
// A_hi*B_hi + A_lo*B_hi and columns [n, 2n) collect A_hi*B_lo; the sum of the
// two blocks is the product.  Two MMAs per K step, A_hi read once.
__device__ __forceinline__ void mma_cat(uint32_t tmem, const uint16_t* A, const uint16_t* Bcat, int n, int K) {
  const uint32_t a_hi = tc::smem_u32(A), a_lo = a_hi + 128u * K * 2u;
  const uint32_t b = tc::smem_u32(Bcat);
  const uint32_t id2 = tc::idesc_bf16(128, 2 * n), id1 = tc::idesc_bf16(128, n);
  for (int ks = 0; ks < K / 16; ++ks) {
    const uint32_t ao = ks * 2u * 128u * 16u, bo = ks * 2u * 2u * (uint32_t)n * 16u;
    const uint64_t ah = tc::make_desc(a_hi + ao, 128 * 16, 128), al = tc::make_desc(a_lo + ao, 128 * 16, 128);
    const uint64_t bc = tc::make_desc(b + bo, 2 * n * 16, 128);  // all 2n rows; the first n are B_hi
    tc::mma_bf16(tmem, ah, bc, id2, ks > 0 ? 1u : 0u);
    tc::mma_bf16(tmem, al, bc, id1, 1u);
  }
}

// (cell, point) enumeration with the cell fastest in groups of 8: lanes of a
// warp cover 8 cells x 4 consecutive points.
__device__ __forceinline__ void cell_point(int idx, int npts, int& c, int& p) {
  const int rest = idx >> 3;
  p = rest % npts;
  c = (rest / npts) * 8 + (idx & 7);
}

// F(qbar + dq) - F(qbar) for the Euler flux, written as telescoped products so
// that no large terms cancel (qbar, dq primitive: rho, u, v, w, p).
__device__ __forceinline__ void euler_flux_delta(const float qb[5], const float dq[5], float dF[3][5]) {
  const float rb = qb[0], dr = dq[0], dp = dq[4];
  const float ub[3] = {qb[1], qb[2], qb[3]}, du[3] = {dq[1], dq[2], dq[3]};
  const float u[3] = {ub[0] + du[0], ub[1] + du[1], ub[2] + du[2]};
  const float g1 = float(GAMMA / (GAMMA - 1.0));
  const float uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  const float d_uu = (u[0] + ub[0]) * du[0] + (u[1] + ub[1]) * du[1] + (u[2] + ub[2]) * du[2];
  const float p = qb[4] + dp;
  const float r = rb + dr;
  const float e = g1 * p + 0.5f * r * uu;                 // rho H
  const float de = g1 * dp + 0.5f * (dr * uu + rb * d_uu);
#pragma unroll
  for (int n = 0; n < 3; ++n) {
    const float dm = dr * u[n] + rb * du[n];              // delta(rho u_n)
    const float mb = rb * ub[n];
    dF[n][0] = dm;
#pragma unroll
    for (int j = 0; j < 3; ++j) dF[n][1 + j] = dm * u[j] + mb * du[j] + (n == j ? dp : 0.f);
    dF[n][4] = du[n] * e + ub[n] * de;
  }
}

// primitives (rho, u, v, w, p) without pressure floor (core/fr_residual/inviscid.py:38-47)
// and T = p / (rho R), with one reciprocal of rho (the mixed form has no bitwise target)
__device__ __forceinline__ void prim_T(const double* U, double q[6]) {
  const double rho = fmax(U[0], 1e-10);
  const double r = 1.0 / rho;
  const double u = U[1] * r, v = U[2] * r, w = U[3] * r;
  const double p = (GAMMA - 1.0) * rho * (U[4] * r - 0.5 * (u * u + v * v + w * w));
  q[0] = rho; q[1] = u; q[2] = v; q[3] = w; q[4] = p;
  q[5] = p * r * (1.0 / R_AIR);
}

__device__ __forceinline__ bool wait_commit(uint64_t* bar, uint32_t& phase, unsigned* status) {
  const bool ok = tc::mbar_wait(bar, phase);
  phase ^= 1u;
  if (!ok) atomicOr(status, (unsigned)DS_TC_TIMEOUT);
  return ok;
}

}  // namespace mxd

// ---------------------------------------------------------------------------
// pre-pass: gradients and face-point extrapolation of one 8-cell tile
// ---------------------------------------------------------------------------
template <int S, int NP>
struct MxPreSmem {
  static constexpr int Sq = pad16(S), NFP = 6 * NP, NB1 = 3 * Sq, NB2MAX = 144;
  static constexpr int oB1 = 0;                        // D3g image (hi|lo)
  static constexpr int oA2 = oB1 + NB1 * Sq * 4;       // E image
  static constexpr int oA1 = oA2 + 128 * Sq * 4;       // gradient inputs, rows phi*8 + c
  static constexpr int oB2 = oA1 + 128 * Sq * 4;       // face-field inputs, rows f*8 + c
  static constexpr int oG = oB2 + NB2MAX * Sq * 4;     // reference-space gradients [c][s][m][phi]
  static constexpr int oQ = oG + MX_PRE_CELLS * S * 12 * 4;  // q and T (FP64) [c][s][6]
  static constexpr int oM = oQ + MX_PRE_CELLS * S * 6 * 8;   // means (FP64) [c][9]
  // the next tile's state rows (stride nv <= 8) and nu_t, copied asynchronously
  // (P1, P2; at P3 the tile's loads are direct: no room)
  static constexpr bool STG = S <= 27;
  static constexpr int oStg = oM + MX_PRE_CELLS * 9 * 8;
  // and the next tile's FP32 inverse-Jacobian rows (float4 x 3 per point), 16-byte aligned
  static constexpr int oInv = (oStg + (STG ? MX_PRE_CELLS * S * 9 * 8 : 0) + 15) / 16 * 16;
  static constexpr int total = oInv + (STG ? MX_PRE_CELLS * S * 48 : 0);
  static constexpr int NCOL = pow2_cols(cmax(NB1, NB2MAX));
};

template <int S, int NP>
__global__ void __launch_bounds__(MX_THREADS, 2)  // 64 registers: two CTAs per SM (tensor memory allows two)
    k_mx_pre(Geom g, MxOps mo, MxBuf mb, const double* __restrict__ U, int nv, const double* __restrict__ nut,
             int visc, int cell_base, int cell_end, unsigned* status) {
  using L = MxPreSmem<S, NP>;
  constexpr int Sq = L::Sq, NFP = L::NFP, C = MX_PRE_CELLS;
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  __shared__ int abort_flag;
  uint16_t* sB1 = reinterpret_cast<uint16_t*>(smem + L::oB1);
  uint16_t* sA2 = reinterpret_cast<uint16_t*>(smem + L::oA2);
  uint16_t* sA1 = reinterpret_cast<uint16_t*>(smem + L::oA1);
  uint16_t* sB2 = reinterpret_cast<uint16_t*>(smem + L::oB2);
  float* sG = reinterpret_cast<float*>(smem + L::oG);
  double* sQ = reinterpret_cast<double*>(smem + L::oQ);
  double* sM = reinterpret_cast<double*>(smem + L::oM);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int FW = mb.FW;
  visc = visc && FW >= 18;
  const int nfw = visc ? 18 : 5;  // fields extrapolated by this call
  const int NB2 = pad16(nfw * C);
  const int ct = cell_type(g, cell_base);

  if (visc) mxd::copy_img(sB1, (ct ? mo.D3g[1] : mo.D3g[0]), L::NB1 * Sq * 4);
  mxd::copy_img(sA2, (ct ? mo.E[1] : mo.E[0]), 128 * Sq * 4);
  // operand padding (K columns s >= S, rows never written) stays zero
  for (int t = tid; t < 128 * Sq * 4 / 16; t += MX_THREADS) reinterpret_cast<uint4*>(sA1)[t] = make_uint4(0, 0, 0, 0);
  for (int t = tid; t < L::NB2MAX * Sq * 4 / 16; t += MX_THREADS)
    reinterpret_cast<uint4*>(sB2)[t] = make_uint4(0, 0, 0, 0);
  if (warp == 0) tc::tmem_alloc(&tbase, L::NCOL);
  if (tid == 0) {
    tc::mbar_init(&bar, 1);
    tc::fence_mbar_init();
    abort_flag = 0;
  }
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tbase;
  uint32_t phase = 0;
  const int ntiles = (cell_end - cell_base + C - 1) / C;

  // asynchronous copies of a tile's contiguous state and nu_t blocks into the
  // staging buffer; issued one tile ahead, so they overlap the tile before
  double* sStg = reinterpret_cast<double*>(smem + L::oStg);
  float4* sInvs = reinterpret_cast<float4*>(smem + L::oInv);
  auto stage = [&](int tl) {
    if constexpr (L::STG) {
      const size_t eb = (size_t)cell_base + (size_t)tl * C;
      const int nn = min(C, cell_end - (int)eb);
      const double* ub = U + eb * S * nv;
      for (int t = tid; t < nn * S * nv; t += MX_THREADS) cp_async8(sStg + t, ub + t);
      if (nut)
        for (int t = tid; t < nn * S; t += MX_THREADS) cp_async8(sStg + C * S * 8 + t, nut + eb * S + t);
      cp_async_commit();
    }
  };
  // the tile's inverse-Jacobian rows: read by the gradient phase, so the next
  // tile's copies are issued only once that phase of the current tile is over
  auto stage_inv = [&](int tl) {
    if constexpr (L::STG) {
      if (visc) {
        const size_t eb = (size_t)cell_base + (size_t)tl * C;
        const int nn = min(C, cell_end - (int)eb);
        const float4* ib = mo.invs + eb * S * 3;
        for (int t = tid; t < nn * S * 3; t += MX_THREADS) cp_async16(sInvs + t, ib + t);
        cp_async_commit();
      }
    }
  };
  if (blockIdx.x < ntiles) {
    stage(blockIdx.x);
    stage_inv(blockIdx.x);
  }

  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int e0 = cell_base + tile * C;
    const int nc = min(C, cell_end - e0);
    if (tid == 0 && tile + (int)gridDim.x < ntiles) {
      // the next tile's remaining inputs (contiguous cell ranges) into L2 while this one runs
      const size_t en = (size_t)cell_base + (size_t)(tile + gridDim.x) * C;
      const size_t nn = min((size_t)C, (size_t)cell_end - en), NS = (size_t)g.N * S;
      if (!L::STG) mxd::prefetch_l2(U, NS * nv * 8, en * S * nv * 8, nn * S * nv * 8);
      if (visc && !L::STG) mxd::prefetch_l2(mo.invs, NS * 48, en * S * 48, nn * S * 48);
      if (nut && !L::STG) mxd::prefetch_l2(nut, NS * 8, en * S * 8, nn * S * 8);
    }
    if constexpr (L::STG) {
      cp_async_wait0();  // this thread's copies of the tile
      __syncthreads();   // everyone's
    }
    // nu_t of the tile's point t = c*S + s
    auto nut_at = [&](int c, int s) -> double {
      return L::STG ? sStg[C * S * 8 + c * S + s] : nut[(size_t)(e0 + c) * S + s];
    };
    // primitives and temperature in FP64
    for (int t = tid; t < C * S; t += MX_THREADS) {
      const int c = t % C, s = t / C;
      double q[6] = {1.0, 0.0, 0.0, 0.0, 1.0, 1.0};
      if (c < nc) mxd::prim_T(L::STG ? sStg + (c * S + s) * nv : U + ((size_t)(e0 + c) * S + s) * nv, q);
#pragma unroll
      for (int v = 0; v < 6; ++v) sQ[(c * S + s) * 6 + v] = q[v];
    }
    __syncthreads();
    // cell means of q (5) and of u, v, w, T (4)
    for (int t = tid; t < C * 9; t += MX_THREADS) {
      const int c = t / 9, k = t % 9;
      const int col = k < 5 ? k : (k < 8 ? k - 4 : 5);
      double acc = 0.0;
      for (int s = 0; s < S; ++s) acc += sQ[(c * S + s) * 6 + col];
      sM[c * 9 + k] = acc * (1.0 / S);
    }
    __syncthreads();
    for (int t = tid; t < C * S; t += MX_THREADS) {
      const int c = t % C, s = t / C;
      const double* q = sQ + (c * S + s) * 6;
      if (c < nc) {
        const float mutf = (visc && nut) ? float(q[0] * nut_at(c, s)) : 0.f;
        float4* o = reinterpret_cast<float4*>(mb.PFm + ((size_t)(e0 + c) * S + s) * 20);
        o[3] = make_float4(mutf, float(q[0]), float(q[1]), float(q[2]));
        o[4] = make_float4(float(q[3]), float(q[4]), 0.f, 0.f);
      }
      if (visc) {
        const double phi[4] = {q[1], q[2], q[3], q[5]};
#pragma unroll
        for (int f = 0; f < 4; ++f)
          mxd::st_split(sA1, 128 * Sq, tc::kmajor_index(f * C + c, s, 128), float(phi[f] - sM[c * 9 + 5 + f]));
        const double mut = (c < nc && nut) ? q[0] * nut_at(c, s) : 0.0;
        mxd::st_split(sB2, NB2 * Sq, tc::kmajor_index(17 * C + c, s, NB2), float(mut));
      }
#pragma unroll
      for (int v = 0; v < 5; ++v)
        mxd::st_split(sB2, NB2 * Sq, tc::kmajor_index(v * C + c, s, NB2), float(q[v] - sM[c * 9 + v]));
    }
    tc::fence_async_smem();
    __syncthreads();
    if (tile + (int)gridDim.x < ntiles) stage(tile + (int)gridDim.x);  // the staging buffer is free again
    if (visc) {
      if (tid == 0) {
        tc::fence_after();
        mxd::mma_split(tmem, sA1, sB1, L::NB1, Sq);
        tc::commit(&bar);
        if (!mxd::wait_commit(&bar, phase, status)) abort_flag = 1;
      }
      __syncthreads();
      if (abort_flag) break;
      tc::fence_after();
      // rows phi*8 + c live in TMEM lanes 0..31: warps 0 and 4 split the columns
      if ((warp & 3) == 0) {
        const int f = lane / C, c = lane % C;
        for (int ch = warp >> 2; ch < L::NB1 / 8; ch += MX_THREADS / 128) {
          float v8[8];
          tc::tmem_ld8(tmem + ch * 8, v8);
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int n = ch * 8 + j, m = n / Sq, s = n % Sq;
            if (s < S) sG[((c * S + s) * 3 + m) * 4 + f] = v8[j];
          }
        }
      }
      __syncthreads();
      // physical gradients (core/fr_operators/gradients.py:23-64) and mu_t
      for (int t = tid; t < C * S; t += MX_THREADS) {
        const int c = t % C, s = t / C;
        float gr[12];
        if (c < nc) {
          const float4* inv = L::STG ? sInvs + (c * S + s) * 3 : mo.invs + ((size_t)(e0 + c) * S + s) * 3;
          float iv[9];
#pragma unroll
          for (int m = 0; m < 3; ++m) {
            const float4 x = L::STG ? inv[m] : __ldg(inv + m);
            iv[m * 3 + 0] = x.x;
            iv[m * 3 + 1] = x.y;
            iv[m * 3 + 2] = x.z;
          }
          const float* gs = sG + (c * S + s) * 12;
#pragma unroll
          for (int f = 0; f < 4; ++f)
#pragma unroll
            for (int n = 0; n < 3; ++n)
              gr[f * 3 + n] = gs[0 * 4 + f] * iv[0 * 3 + n] + gs[1 * 4 + f] * iv[1 * 3 + n] + gs[2 * 4 + f] * iv[2 * 3 + n];
          float4* o = reinterpret_cast<float4*>(mb.PFm + ((size_t)(e0 + c) * S + s) * 20);
          o[0] = make_float4(gr[0], gr[1], gr[2], gr[3]);
          o[1] = make_float4(gr[4], gr[5], gr[6], gr[7]);
          o[2] = make_float4(gr[8], gr[9], gr[10], gr[11]);
        } else {
#pragma unroll
          for (int k = 0; k < 12; ++k) gr[k] = 0.f;
        }
#pragma unroll
        for (int k = 0; k < 12; ++k) mxd::st_split(sB2, NB2 * Sq, tc::kmajor_index((5 + k) * C + c, s, NB2), gr[k]);
      }
      tc::fence_async_smem();
      __syncthreads();
      if (tile + (int)gridDim.x < ntiles) stage_inv(tile + (int)gridDim.x);  // the rows are consumed
    }
    // extrapolation of every field to all face points: D[fp][f*8+c]
    if (tid == 0) {
      tc::fence_after();
      mxd::mma_split(tmem, sA2, sB2, NB2, Sq);
      tc::commit(&bar);
      if (!mxd::wait_commit(&bar, phase, status)) abort_flag = 1;
    }
    __syncthreads();
    if (abort_flag) break;
    tc::fence_after();
    {
      // copy j of the face-point rows (lanes j*128/DUP ...) serves cells
      // [j*C/DUP, (j+1)*C/DUP); the quarters of one copy split its face points
      constexpr int DUP = mx_ext_dup(NFP), QPC = 4 / DUP, CPC = C / DUP;
      const int q4 = warp & 3, j = q4 / QPC, fp = (q4 % QPC) * 32 + lane;
      if ((q4 % QPC) * 32 < NFP) {
        for (int f = warp >> 2; f < nfw; f += MX_THREADS / 128) {
          float vc[CPC];  // this copy's cells only (fixed register indices)
          tc::tmem_ldn<CPC>(tmem + ((uint32_t)(q4 * 32) << 16) + f * 8 + j * CPC, vc);
          if (fp < NFP) {
#pragma unroll
            for (int cc = 0; cc < CPC; ++cc) {
              const int c = j * CPC + cc;
              if (c < nc) {
                const float val = f < 5 ? float(sM[c * 9 + f] + (double)vc[cc]) : vc[cc];
                mb.XF[((size_t)(e0 + c) * FW + f) * NFP + fp] = val;
              }
            }
          }
        }
      }
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
  }
  if constexpr (L::STG) cp_async_wait0();  // copies still in flight after an aborted tile
  tc::fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after();
    tc::tmem_dealloc(tmem, L::NCOL);
  }
}

// ---------------------------------------------------------------------------
// face kernel: one thread per (slot, flux point), fields read at face points
// ---------------------------------------------------------------------------
// The jumps of slot point t from its own face-point fields ow and the other
// side's ot (core/fr_residual/inviscid_kernel_colored.py:86-236,
// core/fr_residual/viscous_flux_kernel.py:335-520)
template <int NP>
__device__ __forceinline__ void mx_face_jump(const Faces& fc, const SlotTable& st, const MxFace& mf, const MxBuf& mb,
                                             const double* __restrict__ hcell, float mu, int visc, int t,
                                             const float (&ow)[18], const float (&ot)[18]) {
  const int sl = t / NP, i = t % NP;
  const int f = st.face[sl];
  const int e = st.cell[sl];
  const int fl = st.flags[sl];
  const bool is_owner = (fl & 1) == 0;
  const bool bnd = (fl & 2) != 0;
  const float side = (fl & 16) ? 1.f : -1.f;
  const double* tnp = fc.tnormal + ((size_t)f * NP + i) * 3;
  const float tn[3] = {float(tnp[0]), float(tnp[1]), float(tnp[2])};
  const float4 ar = mf.arow[t];
  const float a0 = ar.x, a1 = ar.y, a2 = ar.z;
  const float mag = fmaxf(ar.w, 1e-30f);
  float dir[3] = {a0 / mag * side, a1 / mag * side, a2 / mag * side};
  const float sg = is_owner ? 1.f : -1.f;
  const float t0 = sg * tn[0], t1 = sg * tn[1], t2 = sg * tn[2];
  if (dir[0] * t0 + dir[1] * t1 + dir[2] * t2 < 0.5f) { dir[0] = t0; dir[1] = t1; dir[2] = t2; }
  float Fc[5], Fp[3][5];
  ausm_up<float>(ow, ot, dir, Fc);
  euler_flux<float>(ow, Fp);
  float* Jo = mb.Jm + (size_t)t * 10;
#pragma unroll
  for (int v = 0; v < 5; ++v) Jo[v] = Fc[v] * mag * side - (a0 * Fp[0][v] + a1 * Fp[1][v] + a2 * Fp[2][v]);
  if (visc) {
    float qa[5], ga[13];
#pragma unroll
    for (int v = 0; v < 5; ++v) qa[v] = 0.5f * (ow[v] + ot[v]);
#pragma unroll
    for (int k = 0; k < 13; ++k) ga[k] = 0.5f * (ow[5 + k] + ot[5 + k]);
    float Gc[3][5], Go[3][5];
    viscous_flux<float>(qa, ga, ga + 9, mu, ga[12], Gc);
    viscous_flux<float>(ow, ow + 5, ow + 14, mu, ow[17], Go);
    float jv[5];
#pragma unroll
    for (int v = 0; v < 5; ++v)
      jv[v] = (a0 * Gc[0][v] + a1 * Gc[1][v] + a2 * Gc[2][v]) - (a0 * Go[0][v] + a1 * Go[1][v] + a2 * Go[2][v]);
    if (bnd) {
      // interior penalty (core/fr_operators/flux_kernels.py:140-200)
      const float eta = float(C_IP) * (mu + ow[17]) / float(hcell[e]);
      const float scale = eta * ar.w * side;
#pragma unroll
      for (int v = 1; v < 4; ++v) jv[v] += -scale * (ow[v] - ot[v]);
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) Jo[5 + v] = jv[v];
  }
}

template <int S, int NP>
__global__ void __launch_bounds__(256) k_mx_face(Faces fc, Bc bc, SlotTable st, MxFace mf, MxBuf mb,
                                                 const double* __restrict__ hcell, float mu, int visc,
                                                 const int32_t* __restrict__ rest, int n_rest) {
  // slot points not taken by the paired kernel (boundary, interpolated or
  // without a matched partner); all of them when rest is null
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (rest ? n_rest : st.n * NP)) return;
  const int t = rest ? rest[idx] : idx;
  constexpr int NFP = 6 * NP;
  const int sl = t / NP, i = t % NP;
  const int f = st.face[sl];
  const int e = st.cell[sl];
  const int fl = st.flags[sl];
  const bool is_owner = (fl & 1) == 0;
  const bool bnd = (fl & 2) != 0;
  const int ax = (fl >> 2) & 3;
  const int FW = mb.FW;
  const int nf = visc ? 18 : 5;
  float ow[18], ot[18];
  {
    const float* xo = mb.XF + (size_t)e * FW * NFP + (ax * 2 + ((fl & 16) ? 1 : 0)) * NP + i;
#pragma unroll
    for (int k = 0; k < 18; ++k) ow[k] = k < nf ? __ldg(xo + k * NFP) : 0.f;
  }
  const double* tnp = fc.tnormal + ((size_t)f * NP + i) * 3;
  const float tn[3] = {float(tnp[0]), float(tnp[1]), float(tnp[2])};
  if (bnd) {
    float gq[5];
    ghost_state<float>(bc, fc.bc_group[f], ow, tn, gq);
#pragma unroll
    for (int v = 0; v < 5; ++v) ot[v] = gq[v];
#pragma unroll
    for (int k = 5; k < 18; ++k) ot[k] = ow[k];
  } else if (mf.ofp[t] != MX_OFP_GENERAL) {
    // matched rows come from the record's other cell (either source slot may hold them)
    const int oc = is_owner ? fc.neighbor[f] : fc.owner[f];
    const float* xn = mb.XF + (size_t)oc * FW * NFP + mf.ofp[t];
#pragma unroll
    for (int k = 0; k < 18; ++k) ot[k] = k < nf ? __ldg(xn + k * NFP) : 0.f;
  } else {
    // interpolation from the source cells' point fields (sum src0 then src1,
    // zero weights skipped as in core/fr_residual/inviscid_kernel_colored.py:117-121)
#pragma unroll
    for (int k = 0; k < 18; ++k) ot[k] = 0.f;
    for (int src = 0; src < 2; ++src) {
      const int c = src == 0 ? st.c0[sl] : st.c1[sl];
      if (c < 0) continue;
      const double* M = src == 0 ? (is_owner ? fmat(fc.nb_m0, fc.nb_m0i, f, i, NP, S)
                                             : fmat(fc.ow_m0, fc.ow_m0i, f, i, NP, S))
                                 : (is_owner ? fmat(fc.nb_m1, fc.nb_m1i, st.i1[sl], i, NP, S)
                                             : fmat(fc.ow_m1, fc.ow_m1i, st.i1[sl], i, NP, S));
      const float* pf = mb.PFm + (size_t)c * S * 20;
      for (int s = 0; s < S; ++s) {
        const float w = float(__ldg(M + s * NP));
        if (w == 0.f) continue;
        const float4* p4 = reinterpret_cast<const float4*>(pf + s * 20);
        const float4 x3 = __ldg(p4 + 3), x4 = __ldg(p4 + 4);
        ot[0] += w * x3.y; ot[1] += w * x3.z; ot[2] += w * x3.w; ot[3] += w * x4.x; ot[4] += w * x4.y;
        if (visc) {
          const float4 x0 = __ldg(p4), x1 = __ldg(p4 + 1), x2 = __ldg(p4 + 2);
          ot[5] += w * x0.x;  ot[6] += w * x0.y;  ot[7] += w * x0.z;  ot[8] += w * x0.w;
          ot[9] += w * x1.x;  ot[10] += w * x1.y; ot[11] += w * x1.z; ot[12] += w * x1.w;
          ot[13] += w * x2.x; ot[14] += w * x2.y; ot[15] += w * x2.z; ot[16] += w * x2.w;
          ot[17] += w * x3.x;
        }
      }
    }
  }
  mx_face_jump<NP>(fc, st, mf, mb, hcell, mu, visc, t, ow, ot);
}

// Matched interior face points in pairs: slot point t (owner side) and its
// partner t2 (the neighbour side's slot point at the matched face point) read
// the same two face-point rows, own and other swapped; one thread loads them
// once and forms both jumps
template <int S, int NP>
__global__ void __launch_bounds__(256, 3) k_mx_face_pair(Faces fc, Bc bc, SlotTable st, MxFace mf, MxBuf mb,
                                                      const double* __restrict__ hcell, float mu, int visc,
                                                      const int2* __restrict__ pairs, int n_pairs) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_pairs) return;
  constexpr int NFP = 6 * NP;
  const int2 pr = pairs[idx];
  const int t = pr.x, t2 = pr.y;
  const int sl = t / NP, i = t % NP;
  const int f = st.face[sl];
  const int e = st.cell[sl];
  const int fl = st.flags[sl];
  const int ax = (fl >> 2) & 3;
  const int FW = mb.FW;
  const int nf = visc ? 18 : 5;
  const int oc = fc.neighbor[f];
  float ra[18], rb[18];
  {
    const float* xa = mb.XF + (size_t)e * FW * NFP + (ax * 2 + ((fl & 16) ? 1 : 0)) * NP + i;
    const float* xb = mb.XF + (size_t)oc * FW * NFP + mf.ofp[t];
#pragma unroll
    for (int k = 0; k < 18; ++k) {
      ra[k] = k < nf ? __ldg(xa + k * NFP) : 0.f;
      rb[k] = k < nf ? __ldg(xb + k * NFP) : 0.f;
    }
  }
  mx_face_jump<NP>(fc, st, mf, mb, hcell, mu, visc, t, ra, rb);
  mx_face_jump<NP>(fc, st, mf, mb, hcell, mu, visc, t2, rb, ra);
}

// ---------------------------------------------------------------------------
// volume kernel: persistent over C-cell tiles, tensor-core contractions.
// Writes the volume terms RV (N, S, 10) FP32: inviscid -(W*Ft + MD*F(qbar))/det
// (5) and viscous D_3d*Gt/det (5).
// ---------------------------------------------------------------------------
constexpr int MX_VOL_THREADS = 512;

template <int S, int FN, int C>
struct MxVolSmem {
  static constexpr int Sq = pad16(S), Fq = pad16(FN);
  static constexpr bool VP = S <= 27;  // viscous terms built in (P1, P2)
  static constexpr int QS = Fq * 5 + 4;  // floats per cell of the fine-point deviations
  static constexpr int oBc = 0;
  static constexpr int oBW = oBc + Fq * Sq * 4;
  static constexpr int oBD = oBW + Sq * 3 * Fq * 4;
  static constexpr int oR1 = oBD + (VP ? Sq * 3 * Sq * 4 : 0);
  static constexpr int szAc = 128 * Sq * 4, szAD = VP ? 128 * 3 * Sq * 4 : 0, szAW = 128 * 3 * Fq * 4;
  static constexpr int szR1 = cmax(szAc + szAD, szAW);
  static constexpr int oR2 = oR1 + szR1;  // q (FP64) before the first product, then dq, then the RV tile
  static constexpr int szR2 = cmax(cmax(C * QS * 4, C * S * 5 * 8), C * S * 10 * 4);
  static constexpr int oX = oR2 + szR2;
  // doubles: qbar, F(qbar); with VP also det and the metric divergence of the tile
  static constexpr int nX = C * 5 + C * 15 + (VP ? C * S * 4 : 0);
  // the next tile's state rows (stride nv <= 8), 1/det and MD, copied
  // asynchronously (P1, P2; at P3 the tile's loads are direct: no room)
  static constexpr bool STG = VP;
  static constexpr int oStg = oX + nX * 8;
  static constexpr int nStg = STG ? C * S * 12 : 0;
  static constexpr int total = oStg + nStg * 8;
  // TMEM columns: each product holds two column blocks (stacked hi / lo operand)
  static constexpr int cFq = 0, cD3 = 2 * Fq, cW = 2 * Fq + (VP ? 2 * Sq : 0);
  static constexpr int NCOL = pow2_cols(cW + 2 * Sq);
  static_assert(cW + 2 * Sq <= NCOL, "tensor memory columns");
};

template <int S, int FN, int C>
__global__ void __launch_bounds__(MX_VOL_THREADS, 1)
    k_mx_vol(Geom g, MxOps mo, const double* __restrict__ Ucur, int nv, int inviscid_only, float mu,
             const float* __restrict__ PFm, float* __restrict__ RV, int cell_base, int cell_end, unsigned* status) {
  using L = MxVolSmem<S, FN, C>;
  constexpr int Sq = L::Sq, Fq = L::Fq, QS = L::QS, NT = MX_VOL_THREADS;
  static_assert(C % 8 == 0 && 5 * C <= 128, "tile rows (v, c) must fit 128 lanes in groups of 8 cells");
  static_assert(L::NCOL <= 256 && L::total <= 227 * 1024, "tensor memory / shared memory budget");
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  __shared__ int abort_flag;
  uint16_t* sBc = reinterpret_cast<uint16_t*>(smem + L::oBc);
  uint16_t* sBW = reinterpret_cast<uint16_t*>(smem + L::oBW);
  uint16_t* sBD = reinterpret_cast<uint16_t*>(smem + L::oBD);
  uint16_t* sAc = reinterpret_cast<uint16_t*>(smem + L::oR1);
  uint16_t* sAD = reinterpret_cast<uint16_t*>(smem + L::oR1 + L::szAc);
  uint16_t* sAW = reinterpret_cast<uint16_t*>(smem + L::oR1);
  double* sQ = reinterpret_cast<double*>(smem + L::oR2);
  float* sQf = reinterpret_cast<float*>(smem + L::oR2);
  float* sR = reinterpret_cast<float*>(smem + L::oR2);
  double* sQb = reinterpret_cast<double*>(smem + L::oX);  // [c][5]
  double* sFb = sQb + C * 5;                              // [c][n][v] Euler flux at qbar
  double* sDet = sFb + C * 15;                            // [c][s] 1/det (VP)
  double* sMD = sDet + C * S;                             // [c][s][3] (VP)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool visc = L::VP && !inviscid_only;
  const int ct = cell_type(g, cell_base);

  mxd::copy_img(sBc, (ct ? mo.c2f[1] : mo.c2f[0]), Fq * Sq * 4);
  mxd::copy_img(sBW, (ct ? mo.W[1] : mo.W[0]), Sq * 3 * Fq * 4);
  if (visc) mxd::copy_img(sBD, (ct ? mo.D3[1] : mo.D3[0]), Sq * 3 * Sq * 4);
  if (warp == 0) tc::tmem_alloc(&tbase, L::NCOL);
  if (tid == 0) {
    tc::mbar_init(&bar, 1);
    tc::fence_mbar_init();
    abort_flag = 0;
  }
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tbase;
  uint32_t phase = 0;
  const int ntiles = (cell_end - cell_base + C - 1) / C;
  const int q4 = warp & 3;                      // TMEM lane quarter of this warp
  const int lrow = q4 * 32 + lane;              // TMEM lane of this thread
  const uint32_t lane_base = (uint32_t)(q4 * 32) << 16;
  const int wsplit = warp >> 2, nsplit = NT / 128;  // warps sharing a lane quarter split the columns

  // asynchronous copies of a tile's contiguous state, 1/det and MD blocks into
  // the staging buffer; issued one tile ahead, so they overlap the tile before
  double* sStg = reinterpret_cast<double*>(smem + L::oStg);
  auto stage = [&](int tl) {
    if constexpr (L::STG) {
      const size_t eb = (size_t)cell_base + (size_t)tl * C;
      const int nn = min(C, cell_end - (int)eb);
      const double* ub = Ucur + eb * S * nv;
      for (int t = tid; t < nn * S * nv; t += NT) cp_async8(sStg + t, ub + t);
      for (int t = tid; t < nn * S; t += NT) cp_async8(sStg + C * S * 8 + t, mo.rdet + eb * S + t);
      for (int t = tid; t < nn * S * 3; t += NT) cp_async8(sStg + C * S * 9 + t, mo.MD + eb * S * 3 + t);
      cp_async_commit();
    }
  };
  if (blockIdx.x < ntiles) stage(blockIdx.x);

  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int e0 = cell_base + tile * C;
    const int nc = min(C, cell_end - e0);
    if (tid == 0 && tile + (int)gridDim.x < ntiles) {
      // the next tile's remaining inputs (contiguous cell ranges) into L2 while this one runs
      const size_t en = (size_t)cell_base + (size_t)(tile + gridDim.x) * C;
      const size_t nn = min((size_t)C, (size_t)cell_end - en), NS = (size_t)g.N * S;
      mxd::prefetch_l2(mo.adjf, (size_t)g.N * FN * 48, en * FN * 48, nn * FN * 48);
      if (!L::STG) mxd::prefetch_l2(Ucur, NS * nv * 8, en * S * nv * 8, nn * S * nv * 8);
      if (visc) {
        mxd::prefetch_l2(PFm, NS * 80, en * S * 80, nn * S * 80);
        mxd::prefetch_l2(mo.adjs, NS * 48, en * S * 48, nn * S * 48);
      }
    }
    if constexpr (L::STG) {
      cp_async_wait0();  // this thread's copies of the tile
      __syncthreads();   // everyone's
    }
    // ---- primitives (FP64), det and metric divergence of the tile ----
    for (int t = tid; t < C * S; t += NT) {
      const int c = t / S;
      double q[6] = {1.0, 0.0, 0.0, 0.0, 1.0, 1.0};
      if (c < nc) {
        mxd::prim_T(L::STG ? sStg + t * nv : Ucur + ((size_t)e0 * S + t) * nv, q);
        if (L::VP) {
          sDet[t] = sStg[C * S * 8 + t];  // reciprocal: the readouts multiply
          sMD[t * 3 + 0] = sStg[C * S * 9 + t * 3 + 0];
          sMD[t * 3 + 1] = sStg[C * S * 9 + t * 3 + 1];
          sMD[t * 3 + 2] = sStg[C * S * 9 + t * 3 + 2];
        }
      }
#pragma unroll
      for (int v = 0; v < 5; ++v) sQ[t * 5 + v] = q[v];
    }
    __syncthreads();
    if (tile + (int)gridDim.x < ntiles) stage(tile + (int)gridDim.x);  // the staging buffer is free again
    for (int t = tid; t < C * 5; t += NT) {
      const int c = t / 5, v = t % 5;
      double acc = 0.0;
      for (int s = 0; s < S; ++s) acc += sQ[(c * S + s) * 5 + v];
      sQb[t] = acc * (1.0 / S);
    }
    __syncthreads();
    for (int c = tid; c < C; c += NT) {
      double F[3][5];
      euler_flux<double>(sQb + c * 5, F);
#pragma unroll
      for (int n = 0; n < 3; ++n)
#pragma unroll
        for (int v = 0; v < 5; ++v) sFb[c * 15 + n * 5 + v] = F[n][v];
    }
    // ---- A operands: q - qbar at the solution points; contravariant viscous flux ----
    for (int idx = tid; idx < C * Sq; idx += NT) {
      int c, s;
      mxd::cell_point(idx, Sq, c, s);
      const bool live = c < nc && s < S;
#pragma unroll
      for (int v = 0; v < 5; ++v)
        mxd::st_split(sAc, 128 * Sq, tc::kmajor_index(v * C + c, s, 128),
                      live ? float(sQ[(c * S + s) * 5 + v] - sQb[c * 5 + v]) : 0.f);
      if (visc) {
        float Gt[3][5];
#pragma unroll
        for (int m = 0; m < 3; ++m)
#pragma unroll
          for (int v = 0; v < 5; ++v) Gt[m][v] = 0.f;
        if (live) {
          const size_t p = (size_t)(e0 + c) * S + s;
          const float4* pf = reinterpret_cast<const float4*>(PFm + p * 20);
          const float4 g0 = __ldg(pf), g1 = __ldg(pf + 1), g2 = __ldg(pf + 2), g3 = __ldg(pf + 3);
          const float4* am = mo.adjs + p * 3;
          float q[5];
#pragma unroll
          for (int v = 0; v < 5; ++v) q[v] = float(sQ[(c * S + s) * 5 + v]);
          const float gv[9] = {g0.x, g0.y, g0.z, g0.w, g1.x, g1.y, g1.z, g1.w, g2.x};
          const float gT[3] = {g2.y, g2.z, g2.w};
          float G[3][5];
          viscous_flux<float>(q, gv, gT, mu, g3.x, G);
#pragma unroll
          for (int m = 0; m < 3; ++m) {
            const float4 x = __ldg(am + m);
#pragma unroll
            for (int v = 0; v < 5; ++v) Gt[m][v] = x.x * G[0][v] + x.y * G[1][v] + x.z * G[2][v];
          }
        }
#pragma unroll
        for (int m = 0; m < 3; ++m)
#pragma unroll
          for (int v = 0; v < 5; ++v)
            mxd::st_split(sAD, 128 * 3 * Sq, tc::kmajor_index(v * C + c, m * Sq + s, 128), Gt[m][v]);
      }
    }
    // the fine-point adjugate rows of this thread's flux items, loaded now so
    // that their latency overlaps the products and the readout below
    constexpr int NFI = (C * Fq + NT - 1) / NT;
    float4 adf[NFI][3];
#pragma unroll
    for (int k = 0; k < NFI; ++k) {
      const int idx = tid + k * NT;
      int c, i;
      mxd::cell_point(idx, Fq, c, i);
      const bool live = idx < C * Fq && c < nc && i < FN;
      const float4* ad = mo.adjf + ((size_t)(e0 + (live ? c : 0)) * FN + (live ? i : 0)) * 3;
#pragma unroll
      for (int m = 0; m < 3; ++m) adf[k][m] = live ? __ldg(ad + m) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after();
      mxd::mma_cat(tmem + L::cFq, sAc, sBc, Fq, Sq);
      if (visc) mxd::mma_cat(tmem + L::cD3, sAD, sBD, Sq, 3 * Sq);
      tc::commit(&bar);
      if (!mxd::wait_commit(&bar, phase, status)) abort_flag = 1;
    }
    __syncthreads();
    if (abort_flag) break;
    tc::fence_after();
    // ---- fine-point deviations dq = c2f*(q - qbar): TMEM -> shared ----
    if (q4 * 32 < 5 * C) {
      for (int ch = wsplit; ch < Fq / 8; ch += nsplit) {
        float v8[8], w8[8];
        tc::tmem_ld8(tmem + lane_base + L::cFq + ch * 8, v8);
        tc::tmem_ld8(tmem + lane_base + L::cFq + Fq + ch * 8, w8);
        if (lrow < 5 * C) {
          const int v = lrow / C, c = lrow % C;
#pragma unroll
          for (int j = 0; j < 8; ++j) sQf[c * QS + (ch * 8 + j) * 5 + v] = v8[j] + w8[j];
        }
      }
    }
    __syncthreads();
    // ---- contravariant Euler flux deviations at the fine points -> A_W ----
#pragma unroll
    for (int k = 0; k < NFI; ++k) {
      const int idx = tid + k * NT;
      if (idx >= C * Fq) break;
      int c, i;
      mxd::cell_point(idx, Fq, c, i);
      float Ft[3][5];
#pragma unroll
      for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int v = 0; v < 5; ++v) Ft[m][v] = 0.f;
      if (c < nc && i < FN) {
        float qb[5], dq[5], dF[3][5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          qb[v] = float(sQb[c * 5 + v]);
          dq[v] = sQf[c * QS + i * 5 + v];
        }
        mxd::euler_flux_delta(qb, dq, dF);
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          const float4 x = adf[k][m];
#pragma unroll
          for (int v = 0; v < 5; ++v) Ft[m][v] = x.x * dF[0][v] + x.y * dF[1][v] + x.z * dF[2][v];
        }
      }
#pragma unroll
      for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int v = 0; v < 5; ++v)
          mxd::st_split(sAW, 128 * 3 * Fq, tc::kmajor_index(v * C + c, m * Fq + i, 128), Ft[m][v]);
    }
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after();
      mxd::mma_cat(tmem + L::cW, sAW, sBW, Sq, 3 * Fq);
      tc::commit(&bar);
    }
    // viscous divergence while the W product runs (its columns are complete);
    // the dq tile is consumed, so the RV tile reuses its space
    if (q4 * 32 < 5 * C) {
      for (int ch = wsplit; ch < Sq / 8; ch += nsplit) {
        float v8[8], w8[8];
        if (visc) {
          tc::tmem_ld8(tmem + lane_base + L::cD3 + ch * 8, v8);
          tc::tmem_ld8(tmem + lane_base + L::cD3 + Sq + ch * 8, w8);
        }
        if (lrow < 5 * C) {
          const int v = lrow / C, c = lrow % C;
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int s = ch * 8 + j;
            if (s < S && c < nc)
              sR[(c * S + s) * 10 + 5 + v] = visc ? float(double(v8[j] + w8[j]) * sDet[c * S + s]) : 0.f;
          }
        }
      }
    }
    if (tid == 0 && !mxd::wait_commit(&bar, phase, status)) abort_flag = 1;
    __syncthreads();
    if (abort_flag) break;
    tc::fence_after();
    // ---- inviscid volume term: -(W*dFt + MD*F(qbar)) / det ----
    if (q4 * 32 < 5 * C) {
      for (int ch = wsplit; ch < Sq / 8; ch += nsplit) {
        float v8[8], w8[8];
        tc::tmem_ld8(tmem + lane_base + L::cW + ch * 8, v8);
        tc::tmem_ld8(tmem + lane_base + L::cW + Sq + ch * 8, w8);
        if (lrow < 5 * C) {
          const int v = lrow / C, c = lrow % C;
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int s = ch * 8 + j;
            if (s < S && c < nc) {
              const size_t p = (size_t)(e0 + c) * S + s;
              const double* md = L::VP ? sMD + (c * S + s) * 3 : mo.MD + p * 3;
              const double rdj = L::VP ? sDet[c * S + s] : __ldg(mo.rdet + p);
              const double mdf = md[0] * sFb[c * 15 + v] + md[1] * sFb[c * 15 + 5 + v] + md[2] * sFb[c * 15 + 10 + v];
              sR[(c * S + s) * 10 + v] = float(-(double(v8[j] + w8[j]) + mdf) * rdj);
            }
          }
        }
      }
    }
    __syncthreads();
    // coalesced store of the tile's volume terms (cells e0 .. e0+nc are contiguous)
    mxd::copy_f32(RV + (size_t)e0 * S * 10, sR, nc * S * 10);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
  }
  if constexpr (L::STG) cp_async_wait0();  // copies still in flight after an aborted tile
  tc::fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after();
    tc::tmem_dealloc(tmem, L::NCOL);
  }
}

// ---------------------------------------------------------------------------
// update kernel: CPB cells per CTA.  Lifting of the face jumps in ascending
// color order (staged in shared memory), outlier zeroing, then the SSP-RK3
// combination, positivity and filter in FP64 (or the residual-only outputs).
//
// The tile's inputs are contiguous blocks (the cells e0 .. e0+nc of the state,
// step-start state, volume terms, reciprocal det and dt, and the slots of
// those cells' jumps); each arrives in shared memory by one bulk asynchronous
// copy (cp.async.bulk, completion counted in bytes on an mbarrier).  A block
// whose address or size is not a multiple of 16 bytes (odd first cell of a
// range, odd last tile) is copied by 8-byte asynchronous copies instead.
// Shared-memory rows keep the global layout: state rows of n_vars doubles (an
// odd stride, so threads reading consecutive points use distinct banks).
// ---------------------------------------------------------------------------
constexpr int MX_UPD_MAXSLOT = 6;  // slots per cell staged in shared memory (more: read from global)

__host__ __device__ constexpr int align16(int b) { return (b + 15) / 16 * 16; }

template <int S, int NP, int CPB>
struct MxUpdSmem {
  static constexpr int THREADS = 256;
  static constexpr int NVMAX = 7;
  // byte offsets; bulk-copy destinations 16-byte aligned
  static constexpr int bU = 0;                                        // CPB*S*nv doubles
  static constexpr int bU0 = align16(bU + CPB * S * NVMAX * 8);       // step-start state
  static constexpr int bRV = align16(bU0 + CPB * S * NVMAX * 8);      // CPB*S*10 floats
  static constexpr int bRd = align16(bRV + CPB * S * 10 * 4);         // CPB*S doubles
  static constexpr int bDt = align16(bRd + CPB * S * 8);              // CPB*S doubles
  static constexpr int bJ = align16(bDt + CPB * S * 8);               // jumps, 16-byte lead
  static constexpr int bRi = align16(bJ + CPB * MX_UPD_MAXSLOT * NP * 10 * 4 + 16);  // CPB*S*5 doubles
  static constexpr int bRv = bRi + CPB * S * 5 * 8;                   // CPB*S*5 doubles
  static constexpr int bW = bRv + CPB * S * 5 * 8;                    // outliers: CPB*2*OUT_WORK doubles
  static constexpr int bP = bW + CPB * 2 * OUT_WORK * 8;              // 2*CPB*S doubles
  static constexpr int bG = bP + 2 * CPB * S * 8;                     // g_left, g_right (8 doubles)
  static constexpr int bI = bG + 8 * 8;                               // ints
  static constexpr int nI = CPB * MX_UPD_MAXSLOT + CPB + 1 + 6 * S;
  static constexpr int total = bI + nI * 4;
};

namespace mxd {
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   tc::smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(tc::smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool bulk_ok(const void* src, size_t bytes) {
  return ((reinterpret_cast<uintptr_t>(src) | bytes) & 15u) == 0 && bytes > 0;
}
// 8-byte asynchronous copies of a block whose bulk copy is not possible
__device__ __forceinline__ void copy8(void* dst, const void* src, size_t bytes) {
  for (size_t t = threadIdx.x; t < bytes / 8; t += blockDim.x)
    cp_async8(static_cast<char*>(dst) + 8 * t, static_cast<const char*>(src) + 8 * t);
}
}  // namespace mxd

// Outlier zeroing of the mixed update kernel (same rule as
// suppress_outliers_cells, core/fr_operators/troubled_cell.py:346-408): the
// column statistics -- mean |U|, min and max |R|, NaN, and the count against
// the lower bound of the median -- by four threads per column (aligned lane
// groups, combined with shuffles) instead of one.  Reference rows have stride
// ldU.  work >= OUT_WORK doubles per block (block b < nc: sRi of cell b,
// nc + b: sRv of cell b).
template <int S>
__device__ void mx_suppress_outliers(double* sRi, double* sRv, const double* sU, int ldU, int nc, bool visc,
                                     double* work) {
  constexpr int NEED = S - ((S & 1) ? S / 2 : S / 2 - 1);  // elements at or above the (lower) middle rank
  const int nb = nc * (visc ? 2 : 1);
  const int ncol = nb * 5;
  const int n4 = (ncol * 4 + (int)blockDim.x - 1) / (int)blockDim.x * (int)blockDim.x;
  int flagged = 0;
  for (int base = 0; base < n4; base += blockDim.x) {
    const int t = base + threadIdx.x;
    const bool on = t < ncol * 4;
    const int col = on ? (t >> 2) : 0, sub = t & 3;
    const int bb = col / 5, v = col % 5;
    const double* R = bb < nc ? sRi + bb * S * 5 : sRv + (bb - nc) * S * 5;
    const double* Ur = sU + (bb % nc) * S * ldU;
    double acc = 0.0, lo = INFINITY, hi = 0.0;
    int nan = 0;
    if (on)
      for (int s = sub; s < S; s += 4) {
        acc += fabs(Ur[s * ldU + v]);
        const double x = fabs(R[s * 5 + v]);
        lo = fmin(lo, x);
        hi = fmax(hi, x);
        nan |= isnan(x) ? 1 : 0;
      }
#pragma unroll
    for (int o = 1; o < 4; o <<= 1) {
      acc += __shfl_xor_sync(0xffffffffu, acc, o);
      lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
      nan |= __shfl_xor_sync(0xffffffffu, nan, o);
    }
    const double mean = acc / S;
    bool skip = !nan && hi <= 1e4 * fmax(fmax(lo, 1e-9 * mean), 1e-300);
    double bound = lo;
    bool count = !nan && !skip;
    double p = hi * 1e-4;
    if (count) {
      // next double up (p is finite and >= 0 here: its bit pattern plus one)
      for (int it = 0; it < 4 && 1e4 * p < hi; ++it) p = __longlong_as_double(__double_as_longlong(p) + 1);
      count = 1e4 * p >= hi;
    }
    int cnt = 0;
    if (on && count)
      for (int s = sub; s < S; s += 4) cnt += fabs(R[s * 5 + v]) >= p;
#pragma unroll
    for (int o = 1; o < 4; o <<= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (count && cnt >= NEED) {
      skip = true;
      bound = p;
    }
    if (on && sub == 0) {
      double* w = work + bb * OUT_WORK;
      w[5 + v] = mean;
      w[v] = bound;
      w[20 + v] = skip ? 0.0 : 1.0;
      flagged |= !skip;
    }
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

template <int S, int NP, int CPB>
__global__ void __launch_bounds__(MxUpdSmem<S, NP, CPB>::THREADS, 5)
    k_mx_update(Geom g, Ops ops, Faces fc, StageArgs a, const float* __restrict__ RV, const float* __restrict__ Jm,
                const double* __restrict__ rdet) {
  using L = MxUpdSmem<S, NP, CPB>;
  extern __shared__ __align__(128) uint8_t smb[];
  __shared__ uint64_t bar;
  double* sU = reinterpret_cast<double*>(smb + L::bU);
  double* sU0 = reinterpret_cast<double*>(smb + L::bU0);
  float* sRVf = reinterpret_cast<float*>(smb + L::bRV);
  double* sRd = reinterpret_cast<double*>(smb + L::bRd);
  double* sDt = reinterpret_cast<double*>(smb + L::bDt);
  double* sRi = reinterpret_cast<double*>(smb + L::bRi);
  double* sRv = reinterpret_cast<double*>(smb + L::bRv);
  double* work = reinterpret_cast<double*>(smb + L::bW);
  double* part = reinterpret_cast<double*>(smb + L::bP);
  double* sGw = reinterpret_cast<double*>(smb + L::bG);  // [0..3] g_left, [4..7] g_right
  int* sFl = reinterpret_cast<int*>(smb + L::bI);
  int* sPtr = sFl + CPB * MX_UPD_MAXSLOT;
  int* sDfp = sPtr + CPB + 1;
  int* sDco = sDfp + 3 * S;
  const int e0 = a.cell_base + blockIdx.x * CPB;
  const int nc = min(CPB, a.cell_end - e0);
  const int ct = cell_type(g, e0);
  const int nv = a.nv;
  const bool visc = !a.inviscid_only;
  const int tid = threadIdx.x;
  constexpr int N1D = S == 8 ? 2 : (S == 27 ? 3 : 4);
  const int k_beg = fc.slot_ptr[e0], k_end = fc.slot_ptr[e0 + nc];
  const bool staged = (k_end - k_beg) <= CPB * MX_UPD_MAXSLOT;
  // jump block: bytes [jb0, jb1) of Jm rounded out to 16-byte boundaries (the
  // allocation carries 16 bytes of slack); the tile's first jump sits jlead
  // bytes into the staged copy
  const size_t jb0 = (size_t)k_beg * NP * 40, jb1 = (size_t)k_end * NP * 40;
  const size_t ja0 = jb0 & ~size_t(15), ja1 = (jb1 + 15) & ~size_t(15);
  const float* sJ = reinterpret_cast<const float*>(smb + L::bJ + (jb0 - ja0));
  {
    const size_t ub = (size_t)nc * S * nv * 8, pb = (size_t)nc * S * 8, rb = (size_t)nc * S * 40;
    const double* uc = a.Ucur + (size_t)e0 * S * nv;
    const double* u0 = a.U0 + (size_t)e0 * S * nv;
    const float* rv = RV + (size_t)e0 * S * 10;
    const double* rd = rdet + (size_t)e0 * S;
    const double* dt = a.stage >= 0 ? a.dt + (size_t)e0 * S : nullptr;
    const char* jsrc = reinterpret_cast<const char*>(Jm) + ja0;
    const bool bu = mxd::bulk_ok(uc, ub), bu0 = a.stage >= 0 && mxd::bulk_ok(u0, ub), brv = mxd::bulk_ok(rv, rb),
               brd = mxd::bulk_ok(rd, pb), bdt = a.stage >= 0 && mxd::bulk_ok(dt, pb),
               bj = staged && k_end > k_beg;  // rounded out: always aligned
    if (tid == 0) {
      tc::mbar_init(&bar, 1);
      tc::fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) {
      const uint32_t tx = (bu ? ub : 0) + (bu0 ? ub : 0) + (brv ? rb : 0) + (brd ? pb : 0) + (bdt ? pb : 0) +
                          (bj ? ja1 - ja0 : 0);
      mxd::mbar_expect_tx(&bar, tx);
      if (bu) mxd::bulk_g2s(sU, uc, (uint32_t)ub, &bar);
      if (bu0) mxd::bulk_g2s(sU0, u0, (uint32_t)ub, &bar);
      if (brv) mxd::bulk_g2s(sRVf, rv, (uint32_t)rb, &bar);
      if (brd) mxd::bulk_g2s(sRd, rd, (uint32_t)pb, &bar);
      if (bdt) mxd::bulk_g2s(sDt, dt, (uint32_t)pb, &bar);
      if (bj) mxd::bulk_g2s(smb + L::bJ, jsrc, (uint32_t)(ja1 - ja0), &bar);
    }
    if (!bu) mxd::copy8(sU, uc, ub);
    if (a.stage >= 0 && !bu0) mxd::copy8(sU0, u0, ub);
    if (!brv) mxd::copy8(sRVf, rv, rb);
    if (!brd) mxd::copy8(sRd, rd, pb);
    if (a.stage >= 0 && !bdt) mxd::copy8(sDt, dt, pb);
    for (int t = tid; t < 3 * S; t += blockDim.x) {
      sDfp[t] = ops.dist_fp[t];
      sDco[t] = ops.dist_co[t];
    }
    if (tid < N1D) {
      sGw[tid] = ops.g_left[tid];
      sGw[4 + tid] = ops.g_right[tid];
    }
    if (tid <= nc) sPtr[tid] = fc.slot_ptr[e0 + tid];
    if (staged)
      for (int t = tid; t < k_end - k_beg; t += blockDim.x) sFl[t] = a.slot_flags[k_beg + t];
    mxd::cp_async_wait_all();
    uint32_t ph = 0;
    if (!mxd::wait_commit(&bar, ph, a.status)) {
      // the status reports the time-out; wait once more (bounded) so that no
      // copy is still writing this CTA's shared memory when it moves on
      uint32_t ph0 = 0;
      tc::mbar_wait(&bar, ph0);
    }
  }
  __syncthreads();
  // lift the jumps of each cell's slots, ascending color order; two threads
  // per point, one for the inviscid and one for the viscous jumps
  for (int t = tid; t < 2 * nc * S; t += blockDim.x) {
    const int p = t >> 1, half = t & 1;
    if (half && !visc) {
      sRv[p * 5 + 0] = sRv[p * 5 + 1] = sRv[p * 5 + 2] = sRv[p * 5 + 3] = sRv[p * 5 + 4] = 0.0;
      continue;
    }
    const int b = p / S, s = p - b * S;
    double cx[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int k = sPtr[b]; k < sPtr[b + 1]; ++k) {
      const int fl = staged ? sFl[k - k_beg] : a.slot_flags[k];
      const int ax = (fl >> 2) & 3;
      const int fp = sDfp[ax * S + s];
      const double gw = sGw[((fl & 16) ? 4 : 0) + sDco[ax * S + s]];
      const float* Jk = (staged ? sJ + ((k - k_beg) * NP + fp) * 10 : Jm + ((size_t)k * NP + fp) * 10) + 5 * half;
#pragma unroll
      for (int v = 0; v < 5; ++v) cx[v] += gw * double(Jk[v]);
    }
    const double rdj = sRd[p];
    const float* rp = sRVf + p * 10 + 5 * half;
    double* out = half ? sRv : sRi;
    const double sg = half ? 1.0 : -1.0;  // inviscid corrections enter with -g', viscous with +g'
#pragma unroll
    for (int v = 0; v < 5; ++v) out[p * 5 + v] = double(rp[v]) + sg * cx[v] * rdj;
  }
  __syncthreads();
  mx_suppress_outliers<S>(sRi, sRv, sU, nv, nc, visc, work);

  if (a.stage < 0) {
    for (int p = tid; p < nc * S; p += blockDim.x)
      for (int v = 0; v < nv; ++v) {
        const size_t o = ((size_t)e0 * S + p) * nv + v;
        if (a.Rinv) a.Rinv[o] = v < 5 ? sRi[p * 5 + v] : 0.0;
        if (a.Rvisc) a.Rvisc[o] = (v < 5 && visc) ? sRv[p * 5 + v] : 0.0;
      }
    return;
  }
  // RK stage combination + positivity, in place over the state tile (loops
  // over the 8 possible variables, unrolled, so the arrays stay in registers)
  for (int p = tid; p < nc * S; p += blockDim.x) {
    double Lr[8], un[8];
    double sq_sum = 0.0;
#pragma unroll
    for (int v = 0; v < 8; ++v) Lr[v] = v < 5 ? sRi[p * 5 + v] + (visc ? sRv[p * 5 + v] : 0.0) : 0.0;
#pragma unroll
    for (int v = 0; v < 8; ++v)
      if (v < nv) sq_sum += Lr[v] * Lr[v];
    const double dts = sDt[p];
    const double* u0 = sU0 + p * nv;
    double* uc = sU + p * nv;
    if (a.stage == 0) {
#pragma unroll
      for (int v = 0; v < 8; ++v) un[v] = v < nv ? u0[v] + dts * Lr[v] : 0.0;
    } else if (a.stage == 1) {
#pragma unroll
      for (int v = 0; v < 8; ++v) un[v] = v < nv ? (0.75 * u0[v] + 0.25 * uc[v]) + (0.25 * dts) * Lr[v] : 0.0;
    } else {
#pragma unroll
      for (int v = 0; v < 8; ++v)
        un[v] = v < nv ? (1.0 / 3.0 * u0[v] + 2.0 / 3.0 * uc[v]) + (2.0 / 3.0 * dts) * Lr[v] : 0.0;
    }
    // positivity (core/time_integration/positivity.py:13-45), one reciprocal of rho
    const double rho = fmax(un[0], 1e-6);
    un[0] = rho;
    const double rr = 1.0 / rho;
    double vel[3] = {un[1] * rr, un[2] * rr, un[3] * rr};
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
      if (v < nv) uc[v] = un[v];
    part[p] = sq_sum;
    part[CPB * S + p] = Lr[0] * Lr[0];
  }
  __syncthreads();
  // modal filter as one FP64 tensor-core product per tile: rows s, columns
  // (cell, variable) of the first five variables, K = the cell's points; the
  // outputs are assembled in the residual buffers (no longer needed) and
  // stored as one contiguous block
  double* sOut = sRi;  // (nc*S, nv) row-major, fits in sRi + sRv
  dmma_product_f(
      S, 5 * nc, S, ops.ffilt[ct],
      [&](int j, int col) { return sU[((col / 5) * S + j) * nv + col % 5]; },
      [&](int s, int col, double x) { sOut[((col / 5) * S + s) * nv + col % 5] = x; });
  for (int p = tid; p < nc * S; p += blockDim.x)
    for (int v = 5; v < nv; ++v) sOut[p * nv + v] = sU[p * nv + v];
  __syncthreads();
  for (int t = tid; t < nc * S * nv; t += blockDim.x) a.Unext[(size_t)e0 * S * nv + t] = sOut[t];
  if (a.stage == 0 && tid < nc) {
    double acc = 0.0;
    for (int s = 0; s < S; ++s) acc += part[tid * S + s];
    a.norm_part[e0 + tid] = acc;
    double acc_rho = 0.0;
    for (int s = 0; s < S; ++s) acc_rho += part[CPB * S + tid * S + s];
    a.norm_rho_part[e0 + tid] = acc_rho;
    // a non-finite dU/dt anywhere in the cell makes its partial non-finite
    if (!isfinite(acc) && a.status) atomicOr(a.status, (unsigned)DS_NONFINITE);
  }
}

// ---------------------------------------------------------------------------
// set-up kernels of the mixed form
// ---------------------------------------------------------------------------
// own adjugate row at each slot flux point (E * adj, FP64 then rounded) and the
// face point of the other side whose extrapolation row equals the slot's
// interpolation row to tol relative (MX_OFP_GENERAL where none does)
template <int S, int NP>
__global__ void k_mx_match(Geom g, Ops ops, Faces fc, SlotTable st, float4* arow, uint8_t* ofp, double tol) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= st.n * NP) return;
  const int sl = t / NP, i = t % NP;
  const int f = st.face[sl], e = st.cell[sl], fl = st.flags[sl];
  const bool is_owner = (fl & 1) == 0, bnd = (fl & 2) != 0;
  const int ax = (fl >> 2) & 3, sb = (fl & 16) ? 1 : 0;
  const int ct = cell_type(g, e);
  const double* Er = ops.extrap + (((size_t)ct * 3 + ax) * 2 + sb) * NP * S + (size_t)i * S;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int s = 0; s < S; ++s) {
    const double w = Er[s];
    const double* ad = g.adj + ((size_t)e * S + s) * 9 + ax * 3;
    a0 += w * ad[0];
    a1 += w * ad[1];
    a2 += w * ad[2];
  }
  arow[t] = make_float4(float(a0), float(a1), float(a2), float(sqrt(a0 * a0 + a1 * a1 + a2 * a2)));
  if (bnd) {
    ofp[t] = 0;
    return;
  }
  // the other side's interpolation row; the reference may split one cell's
  // row over its two source slots, so same-cell rows are added first
  const int c0 = st.c0[sl], c1 = st.c1[sl];
  const int expect = is_owner ? fc.neighbor[f] : fc.owner[f];
  const bool one_cell = (c0 == expect || c0 < 0) && (c1 == expect || c1 < 0) && (c0 >= 0 || c1 >= 0);
  if (!one_cell) {
    ofp[t] = MX_OFP_GENERAL;
    return;
  }
  const double* M0 =
      c0 >= 0 ? (is_owner ? fmat(fc.nb_m0, fc.nb_m0i, f, i, NP, S) : fmat(fc.ow_m0, fc.ow_m0i, f, i, NP, S)) : nullptr;
  const double* M1 = c1 >= 0 ? (is_owner ? fmat(fc.nb_m1, fc.nb_m1i, st.i1[sl], i, NP, S)
                                         : fmat(fc.ow_m1, fc.ow_m1i, st.i1[sl], i, NP, S))
                             : nullptr;
  const int oax = is_owner ? fc.n_axis[f] : fc.o_axis[f];
  const int osb = (is_owner ? fc.n_side[f] : fc.o_side[f]) > 0.0 ? 1 : 0;
  const int oct = cell_type(g, expect);
  double mmax = 0.0;
  for (int s = 0; s < S; ++s) mmax = fmax(mmax, fabs((M0 ? M0[s * NP] : 0.0) + (M1 ? M1[s * NP] : 0.0)));
  int best = -1;
  double best_err = INFINITY;
  for (int j = 0; j < NP; ++j) {
    const double* Eo = ops.extrap + (((size_t)oct * 3 + oax) * 2 + osb) * NP * S + (size_t)j * S;
    double err = 0.0;
    for (int s = 0; s < S && err <= best_err; ++s)
      err = fmax(err, fabs((M0 ? M0[s * NP] : 0.0) + (M1 ? M1[s * NP] : 0.0) - Eo[s]));
    if (err < best_err) {
      best_err = err;
      best = j;
    }
  }
  ofp[t] = (best >= 0 && best_err <= tol * fmax(mmax, 1e-300)) ? (uint8_t)((oax * 2 + osb) * NP + best)
                                                                 : MX_OFP_GENERAL;
}

// 1 / det per solution point
__global__ void k_mx_rdet(const double* __restrict__ det, size_t n, double* __restrict__ out) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = 1.0 / det[t];
}

// FP32 copies of 3 x 3 metric rows (adjugates, inverse Jacobians: the mixed
// kernels round them to FP32 before use); one row of 3 per float4
__global__ void k_mx_rows_f32(const double* __restrict__ adj_fine, size_t nrows, float4* __restrict__ out) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nrows) return;
  const double* a = adj_fine + t * 3;
  out[t] = make_float4(float(a[0]), float(a[1]), float(a[2]), 0.f);
}

// MD[c,s,n] = sum_{i,m} W[s, i*3+m] adj_fine[c,i,m,n]  (W's columns follow D_fine: i*3+m)
template <int S, int FN>
__global__ void k_mx_md(Geom g, Ops ops, double* MD) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)g.N * S * 3) return;
  const int n = (int)(t % 3);
  const int s = (int)((t / 3) % S);
  const size_t c = t / (3 * S);
  const int ct = cell_type(g, (int)c);
  const double* w = ops.W[ct] + (size_t)s * FN * 3;
  const double* ad = g.adj_fine + c * FN * 9;
  double acc = 0.0;
  for (int i = 0; i < FN; ++i)
    for (int m = 0; m < 3; ++m) acc += w[i * 3 + m] * ad[i * 9 + m * 3 + n];
  MD[t] = acc;
}

template <int S>
__global__ void k_mx_hcell(Geom g, double* hcell) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= g.N) return;
  double vol = 0.0;
  for (int s = 0; s < S; ++s) vol += g.det[(size_t)e * S + s];
  vol /= S;
  double h = pow(vol, 1.0 / 3.0);
  if (h < 1e-300) h = 1e-300;
  hcell[e] = h;
}

}  // namespace afr
