// Fused strong-form Lax-Friedrichs RHS + LSERK4 stage, TMA-pipelined form for sm_100a.
//
// One CTA per SM walks the tile list.  For every tile it streams, with 1-D bulk copies (cp.async.bulk, the
// TMA engine, completion counted in bytes on an mbarrier), the tile's slice of the state, the residual, the
// nine per-node metrics, the four per-face-point face arrays and the gather map into a two-stage shared
// memory ring: while tile t is computed, the copies of tile t+1 are in flight, so HBM streams continuously
// and no registers hold in-flight data.  Only the neighbour traces uP are read with ordinary (L2-cached)
// gathers.  The reference matrices are read through L1 (warp-uniform broadcast loads), which leaves the
// shared memory to the ring.
//
// Every wait on an mbarrier is bounded: if a stage does not complete within the spin limit the kernel
// records kStatusTimeoutCode in the status word, waits (bounded) for the copies it issued, and returns.
#include <cstdint>
#include <type_traits>

#include "dg_kernels.cuh"
#include "tma.cuh"
#include "kernels.hpp"
#include "runner.hpp"

namespace dgk {

// Tile shape of the TMA form: TE elements per tile, RG rows per thread in the element-local products.
template <typename T, int N>
struct TmaShape;
template <> struct TmaShape<double, 1> { static constexpr int TE = 64, RG = 2; };
template <> struct TmaShape<double, 2> { static constexpr int TE = 32, RG = 2; };
template <> struct TmaShape<double, 3> { static constexpr int TE = 16, RG = 3; };
template <> struct TmaShape<double, 4> { static constexpr int TE = 16, RG = 5; };
template <> struct TmaShape<double, 5> { static constexpr int TE = 16, RG = 7; };
template <> struct TmaShape<float, 1> { static constexpr int TE = 64, RG = 2; };
template <> struct TmaShape<float, 2> { static constexpr int TE = 64, RG = 2; };
template <> struct TmaShape<float, 3> { static constexpr int TE = 32, RG = 3; };
template <> struct TmaShape<float, 4> { static constexpr int TE = 32, RG = 5; };
template <> struct TmaShape<float, 5> { static constexpr int TE = 16, RG = 7; };

template <typename T, int N>
struct TmaCfg {
  using O = Order<N>;
  static constexpr int NP = O::NP, NF = O::NF, NPS = O::NPS, NFS = O::NFS;
  static constexpr int TE = TmaShape<T, N>::TE, RG = TmaShape<T, N>::RG;
  static constexpr int G = (NP + RG - 1) / RG;
  static constexpr int THREADS = TE * G;
  // one ring stage: u, resu, 9 metrics (node arrays), nx, ny, nz, Fscale (face arrays), gather map
  static constexpr uint32_t NODE_B = TE * NP * sizeof(T);
  static constexpr uint32_t FACE_B = TE * NF * sizeof(T);
  static constexpr uint32_t GMAP_B = TE * NF * sizeof(int32_t);
  static constexpr uint32_t STAGE_B = 11 * NODE_B + 4 * FACE_B + GMAP_B;
  static constexpr uint32_t WORK_B = (3 * TE * NPS + TE * NFS) * sizeof(T) + NF * sizeof(int32_t);
  static constexpr size_t SMEM = 2 * (size_t)STAGE_B + WORK_B + 2 * sizeof(uint64_t);
  static_assert(NODE_B % 16 == 0 && FACE_B % 16 == 0 && GMAP_B % 16 == 0, "ring slots must stay 16-byte aligned");
};

// Element-local products with the matrix read through L1: rows g*RG .. g*RG+RG-1 of an NR x NC matrix
// (row stride pad_even(NC)) times one vector x of a shared-memory tile; f(x) = x or x^2/2.
template <typename T, int NR, int NC, int RG, bool SQUARE>
__device__ __forceinline__ void rows_matvec_l1(const T *__restrict__ M, const T *xe, int g, T (&acc)[RG]) {
  constexpr int LD = pad_even(NC);
  using T2 = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
#pragma unroll
  for (int r = 0; r < RG; ++r) acc[r] = T(0);
  const int i0 = g * RG;
#pragma unroll 1
  for (int j = 0; j + 1 < NC; j += 2) {
    T x0 = xe[j], x1 = xe[j + 1];
    if (SQUARE) {
      x0 = T(0.5) * x0 * x0;
      x1 = T(0.5) * x1 * x1;
    }
#pragma unroll
    for (int r = 0; r < RG; ++r) {
      const int i = min(i0 + r, NR - 1);  // rows past NR compute a duplicate that is never stored
      const T2 mm = __ldg(reinterpret_cast<const T2 *>(M + i * LD + j));
      acc[r] = fma(mm.x, x0, acc[r]);
      acc[r] = fma(mm.y, x1, acc[r]);
    }
  }
  if (NC & 1) {
    T x0 = xe[NC - 1];
    if (SQUARE) x0 = T(0.5) * x0 * x0;
#pragma unroll
    for (int r = 0; r < RG; ++r) {
      const int i = min(i0 + r, NR - 1);
      acc[r] = fma(__ldg(M + i * LD + NC - 1), x0, acc[r]);
    }
  }
}

template <typename T, int N>
__device__ __forceinline__ void issue_tile(const RhsArgs<T> &A, const Tile &tl, char *stage, uint64_t *bar,
                                           int rhs_only) {
  using C = TmaCfg<T, N>;
  const uint32_t nb = round16((uint32_t)(tl.nelem * C::NP * sizeof(T)));
  const uint32_t fb = round16((uint32_t)(tl.nelem * C::NF * sizeof(T)));
  const uint32_t gb = round16((uint32_t)(tl.nelem * C::NF * sizeof(int32_t)));
  const uint32_t total = (rhs_only ? 10 : 11) * nb + 4 * fb + gb;
  mbar_expect_tx(bar, total);
  bulk_g2s(stage, A.u_in + tl.node_base, nb, bar);
  if (!rhs_only) bulk_g2s(stage + C::NODE_B, A.resu + tl.node_base, nb, bar);
#pragma unroll
  for (int m = 0; m < 9; ++m) bulk_g2s(stage + (2 + m) * C::NODE_B, A.geo[m] + tl.node_base, nb, bar);
#pragma unroll
  for (int m = 0; m < 4; ++m) bulk_g2s(stage + 11 * C::NODE_B + m * C::FACE_B, A.face[m] + tl.face_base, fb, bar);
  bulk_g2s(stage + 11 * C::NODE_B + 4 * C::FACE_B, A.gmap + tl.face_base, gb, bar);
}

template <typename T, int N>
__global__ void __launch_bounds__(TmaCfg<T, N>::THREADS, 1) rhs_stage_tma_kernel(RhsArgs<T> A, int rhs_only) {
  using C = TmaCfg<T, N>;
  constexpr int NP = C::NP, NF = C::NF, NPS = C::NPS, NFS = C::NFS, TE = C::TE, RG = C::RG, THREADS = C::THREADS;
  constexpr int NI = (TE * NP + THREADS - 1) / THREADS;
  constexpr int NJ = (TE * NF + THREADS - 1) / THREADS;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  char *ring = reinterpret_cast<char *>(smem_raw);
  T *sd = reinterpret_cast<T *>(ring + 2 * C::STAGE_B);  // ur, us, ut -> volume -> rhs
  T *sf = sd + 3 * TE * NPS;                              // uP -> surface flux
  int *sfm = reinterpret_cast<int *>(sf + TE * NFS);
  uint64_t *bar = reinterpret_cast<uint64_t *>(sfm + NF + (NF & 1));
  const int tid = threadIdx.x;
  const int e_own = tid % TE, g_own = tid / TE;
  const int G = gridDim.x;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = tid; i < NF; i += THREADS) sfm[i] = A.fmask[i];
  __syncthreads();
  if (tid == 0) {
    if ((int)blockIdx.x < A.ntiles) issue_tile<T, N>(A, A.tiles[blockIdx.x], ring, &bar[0], rhs_only);
    if ((int)blockIdx.x + G < A.ntiles)
      issue_tile<T, N>(A, A.tiles[blockIdx.x + G], ring + C::STAGE_B, &bar[1], rhs_only);
  }
  const T a = A.a, b = A.b, dt = A.dt;
  int k = 0;
  for (int t = blockIdx.x; t < A.ntiles; t += G, ++k) {
    const int s = k & 1;
    const uint32_t parity = (k >> 1) & 1;
    // every thread polls (each needs the acquire of the TMA writes); the give-up decision is CTA-uniform
    const bool ready = mbar_wait_bounded(&bar[s], parity, kSpinLimit);
    if (!__syncthreads_and(ready)) {
      if (tid == 0) atomicExch(A.status, kStatusTimeoutCode);
      // drain: wait (bounded) for every copy this CTA issued and has not consumed, then leave
      mbar_wait_bounded(&bar[s], parity, kSpinLimit);
      if (t + G < A.ntiles) mbar_wait_bounded(&bar[s ^ 1], ((k + 1) >> 1) & 1, kSpinLimit);
      return;
    }
    const Tile tl = A.tiles[t];
    const int ne = tl.nelem, nn = ne * NP, nfc = ne * NF;
    const char *stage = ring + s * C::STAGE_B;
    const T *su = reinterpret_cast<const T *>(stage);
    const T *sr = su + TE * NP;
    const T *sg = sr + TE * NP;  // 9 metric slices, TE*NP apart
    const T *sfc = reinterpret_cast<const T *>(stage + 11 * C::NODE_B);  // 4 face slices, TE*NF apart
    const int32_t *sgm = reinterpret_cast<const int32_t *>(stage + 11 * C::NODE_B + 4 * C::FACE_B);

    // P1: neighbour traces uP (gathers, all issued before any is stored) and ur, us, ut
    {
      T up[NJ];
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const int idx = tid + j * THREADS;
        up[j] = T(0);
        if (idx < nfc) {
          const int32_t src = sgm[idx];
          if (src >= 0 && (int64_t)src < A.n_u_values) up[j] = __ldcg(A.u_in + src);
        }
      }
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const int idx = tid + j * THREADS;
        if (idx < nfc) {
          const int e = idx / NF, q = idx - e * NF;
          sf[e * NFS + q] = up[j];
        }
      }
    }
    if (e_own < ne) {
#pragma unroll 1
      for (int m = 0; m < 3; ++m) {
        T acc[RG];
        if (A.conservative)
          rows_matvec_l1<T, NP, NP, RG, true>(A.Dmat + m * NP * pad_even(NP), su + e_own * NP, g_own, acc);
        else
          rows_matvec_l1<T, NP, NP, RG, false>(A.Dmat + m * NP * pad_even(NP), su + e_own * NP, g_own, acc);
#pragma unroll
        for (int r = 0; r < RG; ++r) {
          const int i = g_own * RG + r;
          if (i < NP) sd[m * TE * NPS + e_own * NPS + i] = acc[r];
        }
      }
    }
    __syncthreads();
    // P2: volume term (metrics from the ring) and the Lax-Friedrichs surface term (face data from the ring)
#pragma unroll
    for (int j = 0; j < NI; ++j) {
      const int idx = tid + j * THREADS;
      if (idx < nn) {
        const int e = idx / NP, i = idx - e * NP;
        const int so = e * NPS + i;
        const T ur = sd[so], us = sd[TE * NPS + so], ut = sd[2 * TE * NPS + so];
        const T ux = sg[0 * TE * NP + idx] * ur + sg[3 * TE * NP + idx] * us + sg[6 * TE * NP + idx] * ut;
        const T uy = sg[1 * TE * NP + idx] * ur + sg[4 * TE * NP + idx] * us + sg[7 * TE * NP + idx] * ut;
        const T uz = sg[2 * TE * NP + idx] * ur + sg[5 * TE * NP + idx] * us + sg[8 * TE * NP + idx] * ut;
        sd[so] = A.conservative ? -(ux + uy + uz) : -su[idx] * (ux + uy + uz);
      }
    }
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
      const int idx = tid + j * THREADS;
      if (idx < nfc) {
        const int e = idx / NF, q = idx - e * NF;
        const T uM = su[e * NP + sfm[q]];
        T uP = sf[e * NFS + q];
        const int32_t src = sgm[idx];
        if (!(src >= 0 && (int64_t)src < A.n_u_values)) {  // rejected index: report it, use the interior trace
          atomicExch(A.status, kStatusBadGather);
          uP = uM;
        }
        const T nsum = sfc[idx] + sfc[TE * NF + idx] + sfc[2 * TE * NF + idx];
        const T fM = T(0.5) * uM * uM * nsum, fP = T(0.5) * uP * uP * nsum;
        const T an = fabs(nsum);
        const T lam = fmax(fabs(uM) * an, fabs(uP) * an);
        const T du = fM - (T(0.5) * (fM + fP) + T(0.5) * lam * (uM - uP));
        sf[e * NFS + q] = sfc[3 * TE * NF + idx] * du;
      }
    }
    __syncthreads();
    // P3: rhs = volume + LIFT (Fscale du)
    if (e_own < ne) {
      T acc[RG];
      rows_matvec_l1<T, NP, NF, RG, false>(A.LIFT, sf + e_own * NFS, g_own, acc);
#pragma unroll
      for (int r = 0; r < RG; ++r) {
        const int i = g_own * RG + r;
        if (i < NP) sd[e_own * NPS + i] += acc[r];
      }
    }
    __syncthreads();
    // P4: LSERK4 stage (or the bare RHS); residual and state from the ring, results streamed out
#pragma unroll
    for (int j = 0; j < NI; ++j) {
      const int idx = tid + j * THREADS;
      if (idx < nn) {
        const int e = idx / NP, i = idx - e * NP;
        const int64_t gi = tl.node_base + idx;
        const T rhs = sd[e * NPS + i];
        if (rhs_only) {
          __stcs(A.rhs_out + gi, rhs);
        } else {
          const T res = a * sr[idx] + dt * rhs;
          __stcs(A.resu + gi, res);
          __stcs(A.u_out + gi, su[idx] + b * res);
        }
      }
    }
    __syncthreads();  // every thread is done with ring stage s
    if (tid == 0 && t + 2 * G < A.ntiles) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue_tile<T, N>(A, A.tiles[t + 2 * G], ring + s * C::STAGE_B, &bar[s], rhs_only);
    }
  }
}

template <typename T, int N>
static bool tma_launch_n(const RhsArgs<T> &A, int rhs_only, int num_sms, cudaStream_t st, LaunchInfo *info) {
  using C = TmaCfg<T, N>;
  auto k = rhs_stage_tma_kernel<T, N>;
  const size_t sm = C::SMEM;
  if (sm > 227 * 1024) return false;
  cuda_check(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm), "smem attr");
  const int grid = std::min(A.ntiles, num_sms);
  if (info) *info = {grid, C::THREADS, (int)sm, 1};
  if (grid > 0) k<<<grid, C::THREADS, sm, st>>>(A, rhs_only);
  return true;
}

template <typename T>
bool launch_rhs_tma(int N, const RhsArgs<T> &A, int rhs_only, int num_sms, cudaStream_t st, LaunchInfo *info) {
  switch (N) {
    case 1: return tma_launch_n<T, 1>(A, rhs_only, num_sms, st, info);
    case 2: return tma_launch_n<T, 2>(A, rhs_only, num_sms, st, info);
    case 3: return tma_launch_n<T, 3>(A, rhs_only, num_sms, st, info);
    case 4: return tma_launch_n<T, 4>(A, rhs_only, num_sms, st, info);
    case 5: return tma_launch_n<T, 5>(A, rhs_only, num_sms, st, info);
    default: return false;
  }
}

template <typename T, int N>
static int tma_te() {
  return TmaCfg<T, N>::SMEM <= 227 * 1024 ? TmaCfg<T, N>::TE : 0;
}

template <typename T>
int tma_tile_elems(int N) {
  switch (N) {
    case 1: return tma_te<T, 1>();
    case 2: return tma_te<T, 2>();
    case 3: return tma_te<T, 3>();
    case 4: return tma_te<T, 4>();
    case 5: return tma_te<T, 5>();
    default: return 0;
  }
}

template bool launch_rhs_tma<double>(int, const RhsArgs<double> &, int, int, cudaStream_t, LaunchInfo *);
template bool launch_rhs_tma<float>(int, const RhsArgs<float> &, int, int, cudaStream_t, LaunchInfo *);
template int tma_tile_elems<double>(int);
template int tma_tile_elems<float>(int);

// ------------------------------------------------------------------------------------------------
// FP64 form with the element-local products on the FP64 tensor path (mma.sync m8n8k4 .f64).
//
// The products OUT = M * U of a tile are small GEMMs: M is NP x NP (Dr, Ds, Dt) or NP x NF (LIFT), U holds
// the TE element vectors of the tile as columns.  Warp w owns rows 8w..8w+7 (one m-tile) of every matrix
// and keeps its A fragments for all k-steps in registers for the whole persistent kernel; per tile it only
// loads B fragments (element values) from the shared-memory ring.  Fragment layouts of m8n8k4 .f64:
// A (8x4, row-major): lane l holds A[l>>2][l&3]; B (4x8, column-major): lane l holds B[l&3][l>>2];
// C/D (8x8): lane l holds C[l>>2][2(l&3)] and C[l>>2][2(l&3)+1].
// ------------------------------------------------------------------------------------------------
template <int N>
struct DmmaShape;
template <> struct DmmaShape<1> { static constexpr int TE = 32; };
template <> struct DmmaShape<2> { static constexpr int TE = 16; };
template <> struct DmmaShape<3> { static constexpr int TE = 8; };
template <> struct DmmaShape<4> { static constexpr int TE = 8; };
template <> struct DmmaShape<5> { static constexpr int TE = 8; };

// CP: compact FP64 form (per element: the kCompactGeo64 constant geometry values instead of the 9 metric and
// 4 face arrays; neighbour traces through the compact connectivity instead of the gather map)
template <int N, bool CP = false>
struct DmmaCfg {
  using O = Order<N>;
  using T = double;
  static constexpr int NP = O::NP, NF = O::NF, NFS = O::NFS;
  static constexpr int TE = DmmaShape<N>::TE;
  static constexpr int MT = (NP + 7) / 8;  // m-tiles (8 rows)
  static constexpr int KT = (NP + 3) / 4;  // k-steps of the derivative matrices
  static constexpr int KL = NF / 4;        // k-steps of LIFT (NF = 4 Nfp)
  static constexpr int NT = TE / 8;        // n-tiles (8 elements)
  static constexpr int CONS = 32 * MT * NT;  // consumer threads: one warp per (m-tile, n-tile)
  static constexpr int THREADS = CONS + 32;  // + one producer warp gathering neighbour traces
  static constexpr uint32_t NODE_B = TE * NP * sizeof(T);
  static constexpr uint32_t FACE_B = TE * NF * sizeof(T);
  static constexpr uint32_t GEOC_B = (uint32_t)TE * kCompactGeo64 * sizeof(T);
  // u, resu, then 9 metrics and 4 face arrays, or the compact geometry
  static constexpr uint32_t STAGE_B = CP ? 2 * NODE_B + GEOC_B : 11 * NODE_B + 4 * FACE_B;
  static constexpr uint32_t GBUF_B = TE * NF * sizeof(T);         // gathered uP of one tile
  // two gathered-uP buffers, two surface-flux buffers (a warp may start the next tile's flux while another
  // still reads this tile's in the LIFT product), the face-point mask
  static constexpr uint32_t WORK_B = 2 * GBUF_B + 2 * TE * NFS * sizeof(T) + NF * sizeof(int32_t);
  static constexpr int FTR = (NF / 4 + 15) & ~15;        // face-order table row: Nfp bytes rounded up to 16
  static constexpr uint32_t FTAB_B = CP ? 256 * FTR : 0;
  static constexpr size_t SMEM = 2 * (size_t)STAGE_B + WORK_B + 10 * sizeof(uint64_t) + FTAB_B;
  static constexpr int MINB = 2 * SMEM <= 227 * 1024 ? 2 : 1;  // co-resident CTAs the launch bounds plan for
  static constexpr int GJ = (TE * NF + 31) / 32;                  // gathers per producer lane and tile
  static_assert(NODE_B % 16 == 0 && FACE_B % 16 == 0 && GBUF_B % 16 == 0 && GEOC_B % 16 == 0,
                "smem slots must stay 16-byte aligned");
  static_assert(TE % 8 == 0 && NF % 4 == 0, "tile must be whole n-tiles");
};

__device__ __forceinline__ void dmma(double &c0, double &c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}


// Barrier among the consumer warps only (named barrier 1), and its AND-reduction form.
template <int CONS>
__device__ __forceinline__ void cons_sync() {
  asm volatile("bar.sync 1, %0;" ::"n"(CONS) : "memory");
}
template <int CONS>
__device__ __forceinline__ bool cons_sync_and(bool p) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred q, o;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.and.pred o, 1, %2, q;\n\t"
      "selp.u32 %0, 1, 0, o;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)p), "n"(CONS)
      : "memory");
  return r != 0;
}

// A tile's stage is filled in two parts with their own barriers: part A (the 9 metrics and 4 face arrays, read
// by the volume products and the flux) and part B (u and resu, read until the update).
template <int N, bool CP>
__device__ __forceinline__ void issue_tile_a(const RhsArgs<double> &A, const Tile &tl, int64_t slot, char *stage,
                                             uint64_t *bar) {
  using C = DmmaCfg<N, CP>;
  if (CP) {  // the compact geometry of the tile's element slots (slots are padded to whole tiles)
    mbar_expect_tx(bar, C::GEOC_B);
    bulk_g2s(stage + 2 * C::NODE_B, A.geoc + slot * kCompactGeo64, C::GEOC_B, bar);
    return;
  }
  const uint32_t nb = round16((uint32_t)(tl.nelem * C::NP * sizeof(double)));
  const uint32_t fb = round16((uint32_t)(tl.nelem * C::NF * sizeof(double)));
  mbar_expect_tx(bar, 9 * nb + 4 * fb);
#pragma unroll
  for (int m = 0; m < 9; ++m) bulk_g2s(stage + (2 + m) * C::NODE_B, A.geo[m] + tl.node_base, nb, bar);
#pragma unroll
  for (int m = 0; m < 4; ++m) bulk_g2s(stage + 11 * C::NODE_B + m * C::FACE_B, A.face[m] + tl.face_base, fb, bar);
}

template <int N, bool CP>
__device__ __forceinline__ void issue_tile_b(const RhsArgs<double> &A, const Tile &tl, char *stage, uint64_t *bar,
                                             int rhs_only) {
  using C = DmmaCfg<N, CP>;
  const uint32_t nb = round16((uint32_t)(tl.nelem * C::NP * sizeof(double)));
  mbar_expect_tx(bar, (rhs_only ? 1 : 2) * nb);
  bulk_g2s(stage, A.u_in + tl.node_base, nb, bar);
  if (!rhs_only) bulk_g2s(stage + C::NODE_B, A.resu + tl.node_base, nb, bar);
}

// Gather indices of one tile's face points for producer lane `lane` (points lane, lane + 32, ...), in two parts
// so the loads can be in flight a tile ahead: dmma_gather_load issues the loads (the gather map entry; in the
// compact form the neighbour's base and the face-order codes from the compact connectivity), and
// dmma_gather_finish adds the point's node from the face-order table (compact form only).
// Points past the tile's last element get 0 (never read).
template <int N, bool CP>
__device__ __forceinline__ void dmma_gather_load(const RhsArgs<double> &A, const Tile &tl, int64_t slot0, int lane,
                                                 int32_t (&src)[DmmaCfg<N, CP>::GJ],
                                                 uint32_t (&code)[DmmaCfg<N, CP>::GJ]) {
  using C = DmmaCfg<N, CP>;
  constexpr int NF = C::NF, GJ = C::GJ;
  const int nfc = tl.nelem * NF;
#pragma unroll
  for (int j = 0; j < GJ; ++j) {
    const int idx = lane + 32 * j;
    src[j] = 0;
    code[j] = 0;
    if (idx < nfc) {
      if (CP) {
        const int e = idx / NF, f = (idx - e * NF) / (NF / 4);
        const int32_t *cn = A.conn + (slot0 + e) * kMixedConnWords;
        src[j] = cn[f];
        code[j] = (uint32_t)cn[4];
      } else {
        src[j] = __ldcs(A.gmap + tl.face_base + idx);
      }
    }
  }
}

template <int N, bool CP>
__device__ __forceinline__ void dmma_gather_finish(const RhsArgs<double> &A, const Tile &tl, const uint8_t *sft,
                                                   int lane, int32_t (&src)[DmmaCfg<N, CP>::GJ],
                                                   const uint32_t (&code)[DmmaCfg<N, CP>::GJ]) {
  if (!CP) return;
  using C = DmmaCfg<N, CP>;
  constexpr int NF = C::NF, GJ = C::GJ, NFP = NF / 4;
  const int nfc = tl.nelem * NF;
  const int ncd = min(A.ncodes, 256);
#pragma unroll
  for (int j = 0; j < GJ; ++j) {
    const int idx = lane + 32 * j;
    if (idx < nfc) {  // the point's face-order code, then the point's node in the neighbour
      const int e = idx / NF, q = idx - e * NF, f = q / NFP, p = q - f * NFP;
      const int cd = min((int)((code[j] >> (8 * f)) & 0xffu), ncd - 1);
      src[j] += sft[cd * C::FTR + p];
    }
  }
}

// Warp-specialized CTA.  Producer warp: for tile k it reads the tile's gather map and the neighbour traces uP
// from global memory (one batch of loads per lane), writes them to gbuf[k & 1] and signals gready; it runs up
// to two tiles ahead, gated by gfree.  Consumer warps: wait for the TMA stage and gready, then
// (a) [Dr;Ds;Dt] * U on the tensor path with the metrics applied in the epilogue (volume terms stay in
// registers), (b) the Lax-Friedrichs flux of their face points, (c) LIFT * flux on the tensor path with the
// LSERK4 update in the epilogue, streamed to HBM.  One consumer barrier per tile, after the flux (it also
// AND-reduces the waits' outcome, so a timed-out wait ends every consumer there); the end of a tile is a
// counter instead: each consumer warp adds one when it has read the slot's u and resu, and the last one issues
// the slot's refill, so a warp goes on to the next tile without waiting for the others.  The flux buffer
// alternates with the slot: warps are at most one tile apart (the next barrier needs all of them).
template <int N, bool CP>
__global__ void __launch_bounds__(DmmaCfg<N, CP>::THREADS, DmmaCfg<N, CP>::MINB)
    rhs_stage_dmma_kernel(RhsArgs<double> A, int rhs_only) {
  using C = DmmaCfg<N, CP>;
  using T = double;
  constexpr int NP = C::NP, NF = C::NF, NFS = C::NFS, TE = C::TE, CONS = C::CONS;
  constexpr int KT = C::KT, KL = C::KL, MT = C::MT, GJ = C::GJ;
  constexpr int LDD = pad_even(NP), LDL = pad_even(NF);
  constexpr int NJ = (TE * NF + CONS - 1) / CONS;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  char *ring = reinterpret_cast<char *>(smem_raw);
  T *gbuf = reinterpret_cast<T *>(ring + 2 * C::STAGE_B);  // [2][TE*NF] gathered uP
  T *sf2 = gbuf + 2 * TE * NF;                               // [2][TE*NFS] surface flux of the tile
  int *sfm = reinterpret_cast<int *>(sf2 + 2 * TE * NFS);
  uint64_t *bar = reinterpret_cast<uint64_t *>(sfm + NF);    // fullA[2], gready[2], gfree[2], fullB[2]
  uint64_t *full = bar, *gready = bar + 2, *gfree = bar + 4, *fullb = bar + 6;
  int *done = reinterpret_cast<int *>(bar + 8);          // [2] consumer warps done with the slot's u and resu
  uint8_t *sft = reinterpret_cast<uint8_t *>(bar + 10);  // compact form: face-order rows of C::FTR bytes
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int G = gridDim.x;
  if (tid == 0) {
    for (int i = 0; i < 8; ++i) mbar_init(&bar[i], 1);
    done[0] = done[1] = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = tid; i < NF; i += C::THREADS) sfm[i] = A.fmask[i];
  if (CP) {
    constexpr int NFP = NF / 4;
    for (int i = tid; i < min(A.ncodes, 256) * C::FTR; i += C::THREADS) {
      const int row = i / C::FTR, col = i - row * C::FTR;
      sft[i] = col < NFP ? A.ftab[row * NFP + col] : 0;
    }
  }
  __syncthreads();

  if (tid >= CONS) {
    // ---------------- producer warp: neighbour traces ----------------
    // Software-pipelined over the CTA's tiles: while the traces of tile t are gathered, the loads of tile t + G's
    // gather indices (from its descriptor, loaded one tile earlier) and of tile t + 2G's descriptor are in
    // flight, so a tile costs one dependent round trip to memory instead of three (64^3 x 6 order 4: the stage
    // went from 2.17 to 1.94 ms).
    Tile tl = A.tiles[blockIdx.x], tn = {};
    int64_t sl = CP ? A.tile_slot[blockIdx.x] : 0, sn = 0;
    if (blockIdx.x + G < A.ntiles) {
      tn = A.tiles[blockIdx.x + G];
      if (CP) sn = A.tile_slot[blockIdx.x + G];
    }
    // The compact form's index loads feed arithmetic (the face-order table) at once, so it is not pipelined: its
    // loads are issued after the wait for the tile's buffer (pipelined, the compact stage ran 5% slower).
    int32_t src[GJ];
    uint32_t code[GJ];
    if (!CP) dmma_gather_load<N, CP>(A, tl, sl, lane, src, code);
    int k = 0;
    for (int t = blockIdx.x; t < A.ntiles; t += G, ++k) {
      const int s = k & 1;
      if (k >= 2 && !mbar_wait_bounded(&gfree[s], ((k >> 1) - 1) & 1, kSpinLimit)) {
        if (lane == 0) atomicExch(A.status, kStatusTimeoutCode);
        return;  // consumers time out on gready and leave as well
      }
      if (CP) dmma_gather_load<N, CP>(A, tl, sl, lane, src, code);
      dmma_gather_finish<N, CP>(A, tl, sft, lane, src, code);
      const int nfc = tl.nelem * NF;
      T up[GJ];
#pragma unroll
      for (int j = 0; j < GJ; ++j) {
        const int idx = lane + 32 * j;
        up[j] = 0.0;
        if (idx < nfc) {
          if (src[j] >= 0 && (int64_t)src[j] < A.n_u_values) {
            up[j] = __ldcg(A.u_in + src[j]);
          } else {  // rejected index: report it and use the interior trace
            atomicExch(A.status, kStatusBadGather);
            const int e = idx / NF, q = idx - e * NF;
            up[j] = A.u_in[tl.node_base + e * NP + sfm[q]];
          }
        }
      }
      // in flight with the gathers: the next tile's indices and the descriptor after it
      Tile tnn = {};
      int64_t snn = 0;
      if (t + 2 * G < A.ntiles) {
        tnn = A.tiles[t + 2 * G];
        if (CP) snn = A.tile_slot[t + 2 * G];
      }
      if (!CP && t + G < A.ntiles) dmma_gather_load<N, CP>(A, tn, sn, lane, src, code);
      T *g = gbuf + s * TE * NF;
#pragma unroll
      for (int j = 0; j < GJ; ++j) {
        const int idx = lane + 32 * j;
        if (idx < nfc) g[idx] = up[j];
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&gready[s]);
      tl = tn;
      sl = sn;
      tn = tnn;
      sn = snn;
    }
    return;
  }

  // ---------------- consumer warps ----------------
  const int mt = warp % MT, nt = warp / MT;
  const int arow = mt * 8 + (lane >> 2);  // output row of this lane (A row, C row)
  const int acol = lane & 3;              // column within a k-step (A col, B row)
  const int be = nt * 8 + (lane >> 2);    // element of this lane's B fragment
  const int ce = nt * 8 + 2 * acol;       // first of the two elements of this lane's C fragment
  // A fragments of Dr, Ds, Dt and LIFT for this warp's m-tile, resident for the kernel's lifetime
  T aD[3][KT], aL[KL];
#pragma unroll
  for (int m = 0; m < 3; ++m)
#pragma unroll
    for (int kk = 0; kk < KT; ++kk) {
      const int j = 4 * kk + acol;
      aD[m][kk] = (arow < NP && j < NP) ? A.Dmat[(m * NP + arow) * LDD + j] : 0.0;
    }
#pragma unroll
  for (int kk = 0; kk < KL; ++kk) aL[kk] = arow < NP ? A.LIFT[arow * LDL + 4 * kk + acol] : 0.0;
  if (tid == 0) {
    for (int j = 0; j < 2; ++j)
      if ((int)blockIdx.x + j * G < A.ntiles) {
        const Tile tj = A.tiles[blockIdx.x + j * G];
        issue_tile_a<N, CP>(A, tj, CP ? A.tile_slot[blockIdx.x + j * G] : 0, ring + j * C::STAGE_B, &full[j]);
        issue_tile_b<N, CP>(A, tj, ring + j * C::STAGE_B, &fullb[j], rhs_only);
      }
  }
  const T a = A.a, b = A.b, dt = A.dt;
  constexpr int NW = CONS / 32;  // consumer warps
  // tile descriptors in registers: this tile's and the next were loaded in earlier iterations; tile t + 2G's
  // (read by the refills mid-tile) is loaded at the top of the iteration, before the waits
  Tile tcur = A.tiles[blockIdx.x];
  Tile tnext = blockIdx.x + G < A.ntiles ? A.tiles[blockIdx.x + G] : Tile{};
  int k = 0;
  for (int t = blockIdx.x; t < A.ntiles; t += G, ++k) {
    const int s = k & 1;
    const uint32_t parity = (k >> 1) & 1;
    const bool has2 = t + 2 * G < A.ntiles;
    Tile t2 = {};
    int64_t slot2 = 0;
    if (has2) {
      t2 = A.tiles[t + 2 * G];
      if (CP) slot2 = A.tile_slot[t + 2 * G];
    }
    // a wait that gives up leaves the slot unread: the tile is computed from whatever the slot holds (every
    // index stays inside the shared-memory buffers) and the barrier after the flux ends all consumers
    const bool ready = mbar_wait_bounded(&full[s], parity, kSpinLimit) &&
                       mbar_wait_bounded(&fullb[s], parity, kSpinLimit) &&
                       mbar_wait_bounded(&gready[s], parity, kSpinLimit);
    const Tile tl = tcur;
    const int ne = tl.nelem, nfc = ne * NF;
    const char *stage = ring + s * C::STAGE_B;
    const T *su = reinterpret_cast<const T *>(stage);
    const T *sr = su + TE * NP;
    const T *sg = sr + TE * NP;  // per-node metrics; in the compact form the per-element geometry
    const T *sfc = reinterpret_cast<const T *>(stage + 11 * C::NODE_B);
    const T *g = gbuf + s * TE * NF;
    T *sf = sf2 + s * TE * NFS;

    // (a) ur, us, ut on the tensor path; two interleaved accumulator chains per matrix
    T vol[2] = {0.0, 0.0};
    {
      T c[3][2][2];
#pragma unroll
      for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int h = 0; h < 2; ++h) c[m][h][0] = c[m][h][1] = 0.0;
#pragma unroll
      for (int kk = 0; kk < KT; ++kk) {
        const int j = 4 * kk + acol;
        T bv = (j < NP && be < ne) ? su[be * NP + j] : 0.0;
        if (A.conservative) bv = 0.5 * bv * bv;
#pragma unroll
        for (int m = 0; m < 3; ++m) dmma(c[m][kk & 1][0], c[m][kk & 1][1], aD[m][kk], bv);
      }
      // epilogue: metrics at (element, node) and the volume term of the reference's quasi-linear form
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int e = ce + h;
        if (arow < NP && e < ne) {
          const int o = e * NP + arow;
          const T ur = c[0][0][h] + c[0][1][h], us = c[1][0][h] + c[1][1][h], ut = c[2][0][h] + c[2][1][h];
          T m9[9];
#pragma unroll
          for (int m = 0; m < 9; ++m) m9[m] = CP ? sg[e * kCompactGeo64 + m] : sg[m * TE * NP + o];
          const T ux = m9[0] * ur + m9[3] * us + m9[6] * ut;
          const T uy = m9[1] * ur + m9[4] * us + m9[7] * ut;
          const T uz = m9[2] * ur + m9[5] * us + m9[8] * ut;
          vol[h] = A.conservative ? -(ux + uy + uz) : -su[o] * (ux + uy + uz);
        }
      }
    }
    // (b) Lax-Friedrichs flux of this thread's face points
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
      const int idx = tid + j * CONS;
      if (idx < nfc) {
        const int e = idx / NF, q = idx - e * NF;
        const T uM = su[e * NP + sfm[q]];
        const T uP = g[idx];
        const T *gf = sg + e * kCompactGeo64 + 9 + 4 * (q / (NF / 4));  // compact form: the face's nx ny nz Fscale
        const T nsum = CP ? gf[0] + gf[1] + gf[2] : sfc[idx] + sfc[TE * NF + idx] + sfc[2 * TE * NF + idx];
        const T fM = 0.5 * uM * uM * nsum, fP = 0.5 * uP * uP * nsum;
        const T an = fabs(nsum);
        const T lam = fmax(fabs(uM) * an, fabs(uP) * an);
        const T du = fM - (0.5 * (fM + fP) + 0.5 * lam * (uM - uP));
        sf[e * NFS + q] = (CP ? gf[3] : sfc[3 * TE * NF + idx]) * du;
      }
    }
    if (!cons_sync_and<CONS>(ready)) {
      if (tid == 0) atomicExch(A.status, kStatusTimeoutCode);
      // the copies in flight land before the CTA goes: this tile's and the next tile's (the next tile's part B
      // was issued when every consumer had finished the previous tile, before this barrier)
      mbar_wait_bounded(&full[s], parity, kSpinLimit);
      mbar_wait_bounded(&fullb[s], parity, kSpinLimit);
      if (t + G < A.ntiles) {
        mbar_wait_bounded(&full[s ^ 1], ((k + 1) >> 1) & 1, kSpinLimit);
        mbar_wait_bounded(&fullb[s ^ 1], ((k + 1) >> 1) & 1, kSpinLimit);
      }
      return;
    }
    if (tid == 0) {
      mbar_arrive(&gfree[s]);  // the gathered traces of this tile are consumed
      // the metrics and face arrays of stage s are consumed too: tile t + 2G's part A streams in during (c)
      if (has2) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue_tile_a<N, CP>(A, t2, slot2, ring + s * C::STAGE_B, &full[s]);
      }
    }
    // (c) LIFT * flux on the tensor path, LSERK4 update in the epilogue
    {
      T c[3][2];
#pragma unroll
      for (int h = 0; h < 3; ++h) c[h][0] = c[h][1] = 0.0;
#pragma unroll
      for (int kk = 0; kk < KL; ++kk) {
        const T bv = be < ne ? sf[be * NFS + 4 * kk + acol] : 0.0;
        dmma(c[kk % 3][0], c[kk % 3][1], aL[kk], bv);
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int e = ce + h;
        if (arow < NP && e < ne) {
          const int o = e * NP + arow;
          const int64_t gi = tl.node_base + o;
          const T rhs = vol[h] + (c[0][h] + c[1][h] + c[2][h]);
          if (rhs_only) {
            __stcs(A.rhs_out + gi, rhs);
          } else {
            const T res = a * sr[o] + dt * rhs;
            __stcs(A.resu + gi, res);
            __stcs(A.u_out + gi, su[o] + b * res);
          }
        }
      }
    }
    // this warp has read the slot's u and resu (its loads returned: their values are in the stores above); the
    // last consumer warp to get here refills the slot's part B.  Slot s's counter is next touched by tile
    // t + 2G, which no warp reaches before every warp passed tile t + G's barrier, after this reset.
    __syncwarp();
    if (lane == 0) {
      __threadfence_block();
      if (atomicAdd(&done[s], 1) == NW - 1) {
        done[s] = 0;
        __threadfence_block();
        if (has2) {
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          issue_tile_b<N, CP>(A, t2, ring + s * C::STAGE_B, &fullb[s], rhs_only);
        }
      }
    }
    // rotate the descriptors at the end of the tile, where t2's load has long returned
    tcur = tnext;
    tnext = t2;
  }
}

template <int N, bool CP>
static bool dmma_launch_n(const RhsArgs<double> &A, int rhs_only, int num_sms, cudaStream_t st, LaunchInfo *info) {
  using C = DmmaCfg<N, CP>;
  if (C::SMEM > 227 * 1024) return false;
  auto k = rhs_stage_dmma_kernel<N, CP>;
  cuda_check(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM), "smem attr");
  int per = 0;
  cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, C::THREADS, C::SMEM), "occupancy");
  per = std::max(1, per);
  const int grid = std::min(A.ntiles, per * num_sms);
  if (info) *info = {grid, C::THREADS, (int)C::SMEM, per};
  if (grid > 0) k<<<grid, C::THREADS, C::SMEM, st>>>(A, rhs_only);
  return true;
}

// Compact FP64 geometry of the compact form: per element slot the node-0 metrics and, per face, the first face
// point's nx, ny, nz and Fscale; an element whose values vary over its nodes or face points by more than 1e-6
// of the row's scale (the mixed stage's rule: node-to-node round-off of the FP64 metrics, where a curved
// element differs by O(h)) is counted in *bad (the form needs straight-sided elements).
__global__ void compact_geo64_kernel(CompactGeoArgs<double> g, double *out) {
  const int nfp = g.nf / 4;
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < g.elem_total;
       x += (int64_t)gridDim.x * blockDim.x) {
    int p = 0;
    while (p + 1 < g.npart && g.elem_prefix[p + 1] <= x) ++p;
    const int64_t le = x - g.elem_prefix[p];
    const int64_t nb = g.node_off[p] + le * g.np, fb = g.face_off[p] + le * g.nf;
    double *o = out + (g.slot_prefix[p] + le) * kCompactGeo64;
    bool bad = false;
    for (int d = 0; d < 3; ++d) {
      double scale = 0.0;
      for (int q = 0; q < 3; ++q) scale = fmax(scale, fabs(g.geo[3 * d + q][nb]));
      for (int q = 0; q < 3; ++q) {
        const int m = 3 * d + q;
        const double v = g.geo[m][nb];
        for (int i = 1; i < g.np; ++i) bad |= !(fabs(g.geo[m][nb + i] - v) <= 1e-6 * scale);
        o[m] = v;
      }
    }
    for (int f = 0; f < 4; ++f) {
      const int64_t q0 = fb + f * nfp;
      const double ns = fmax(fabs(g.face[0][q0]), fmax(fabs(g.face[1][q0]), fabs(g.face[2][q0])));
      for (int c = 0; c < 4; ++c) {
        const double v = g.face[c][q0], sc = c < 3 ? ns : fabs(v);
        for (int q = 1; q < nfp; ++q) bad |= !(fabs(g.face[c][q0 + q] - v) <= 1e-6 * sc);
        o[9 + 4 * f + c] = v;
      }
    }
    if (bad) atomicAdd(g.bad, 1);
  }
}

void launch_compact_geo64(const CompactGeoArgs<double> &g, double *out, cudaStream_t st) {
  compact_geo64_kernel<<<592, 256, 0, st>>>(g, out);
  cuda_check(cudaGetLastError(), "compact_geo64_kernel launch");
}

bool launch_rhs_dmma(int N, const RhsArgs<double> &A, int rhs_only, int num_sms, cudaStream_t st, LaunchInfo *info) {
  switch (N) {
    case 1: return A.geoc ? dmma_launch_n<1, true>(A, rhs_only, num_sms, st, info)
                   : dmma_launch_n<1, false>(A, rhs_only, num_sms, st, info);
    case 2: return A.geoc ? dmma_launch_n<2, true>(A, rhs_only, num_sms, st, info)
                   : dmma_launch_n<2, false>(A, rhs_only, num_sms, st, info);
    case 3: return A.geoc ? dmma_launch_n<3, true>(A, rhs_only, num_sms, st, info)
                   : dmma_launch_n<3, false>(A, rhs_only, num_sms, st, info);
    case 4: return A.geoc ? dmma_launch_n<4, true>(A, rhs_only, num_sms, st, info)
                   : dmma_launch_n<4, false>(A, rhs_only, num_sms, st, info);
    case 5: return A.geoc ? dmma_launch_n<5, true>(A, rhs_only, num_sms, st, info)
                   : dmma_launch_n<5, false>(A, rhs_only, num_sms, st, info);
    default: return false;
  }
}

template <int N>
static int dmma_te() {
  return DmmaCfg<N>::SMEM <= 227 * 1024 ? DmmaCfg<N>::TE : 0;
}

int dmma_tile_elems(int N) {
  switch (N) {
    case 1: return dmma_te<1>();
    case 2: return dmma_te<2>();
    case 3: return dmma_te<3>();
    case 4: return dmma_te<4>();
    case 5: return dmma_te<5>();
    default: return 0;
  }
}

}  // namespace dgk
