// Mixed-precision stage with its element-local products on the tensor cores (tcgen05, sm_100a), orders 1..4.
//
// Same arithmetic contract as rhs_stage_mixed_kernel (mixed.cu): the state is a compensated FP32 pair
// (u = hi + lo), the residual FP32; the derivative operand is w minus its linear vertex
// interpolant (w = u or u^2/2), whose exact derivative is added back; the Lax-Friedrichs flux is formed in
// FP32.  The two products per element, D{r,s,t} dw and LIFT flux, run as GEMMs over tiles of up to 128
// elements:
//
//   acc_V[e][3i+d] = sum_j dw[e][j] D_d[i][j]      M = 128 elements, N = rup16(3 Np), K = rup16(Np)
//   acc_L[e][i]    = sum_m fl[e][m] LIFT[i][m]     M = 128 elements, N = rup16(Np),   K = 4 rup8(Nfp)
//                                                  (face-major K, each face's points padded to 8)
//
// with elements on the MMA's M dimension, so that TMEM lane e holds element e's operand rows and outputs and
// the threads that own element e write and read them.  Every operand is split into three BF16 parts,
// x = x0 + x1 + x2 (x0 = bf16(x), x1 = bf16(x - x0), x2 = bf16(x - x0 - x1), about 24 significant bits), and
// a product keeps the six terms a_p b_q with p + q <= 2, all accumulated in one FP32 TMEM accumulator: the
// products carry FP32-level rounding (the dropped terms are below 2^-24 of the product).
//
// CTA: one producer warp streams each tile's state (hi, lo, resu), compact geometry, tile-local connectivity
// and halo list (the faces whose neighbour lies outside the tile, listed per tile by the host) into a 2-slot
// ring with 1-D bulk copies and writes finished slots back with bulk stores; one MMA warp issues the GEMMs
// with operand A read from tensor memory and operand B (D and LIFT, split) from shared memory, where it stays
// for the whole launch; CW consumer warps hold CW / 4 threads per element (warps w, w + 4, ... share the TMEM
// lane quarter w mod 4 and split the element's nodes in 8-wide chunks and its faces).  Per tile: the consumer
// threads read their faces' neighbour traces from the slot (inside the tile, or the halo), store the split dw
// into TMEM and arrive on an mbarrier, on which the MMA warp issues the volume GEMM; they form the flux
// meanwhile, store it into its own TMEM columns and arrive again for the LIFT GEMM; while the MMAs run they
// gather the next tile's halo values into the other slot with 4-byte asynchronous copies (a few per thread);
// then they read both accumulators and finish the stage (the compensated update in error-free FP32
// arithmetic) into the slot.  No barrier among the consumers within a tile.  Every wait is bounded; a failed
// wait sets the status word and the CTA leaves after draining its copies and MMAs; TMEM is always freed.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>

#include "dg_kernels.cuh"
#include "kernels.hpp"
#include "runner.hpp"
#include "tcgen05.cuh"
#include "tma.cuh"

namespace dgk {

namespace {

constexpr int kTmTE = 128;    // elements per tile at most (the MMA's M)
constexpr int kTmHalo = 256;  // halo faces per tile at most (even)
constexpr int kTmCols = 512;  // TMEM columns: accumulators, then the split A operands

template <int N>
struct TmCfg {
  using O = Order<N>;
  static constexpr int NP = O::NP, NFP = O::NFP, NF = O::NF;
  // LIFT's K runs face-major, each face padded to KF columns: column f KF + p holds face f's point p
  static constexpr int KF = (NFP + 7) & ~7;
  static constexpr int KV = rup16(NP), KL = rup16(4 * KF), NV = rup16(3 * NP), NL = rup16(NP);
  static constexpr uint32_t BV_PART = (uint32_t)NV * KV * 2, BL_PART = (uint32_t)NL * KL * 2;
  // slot layout (bytes from the slot's start): hi, lo, resu, geometry, tile-local connectivity, halo list,
  // halo values (NFP floats per halo face, in the face's point order)
  static constexpr uint32_t NODE_B = (uint32_t)kTmTE * NP * 4;
  static constexpr uint32_t GEO_B = (uint32_t)kTmTE * kMixedGeoWords * 4;
  static constexpr uint32_t TC_B = (uint32_t)kTmTE * 4 * 4;
  static constexpr uint32_t HL_B = (uint32_t)kTmHalo * 8;
  static constexpr uint32_t HV_B = round16((uint32_t)kTmHalo * NFP * 4);
  static constexpr uint32_t S_GEO = 3 * NODE_B, S_TC = S_GEO + GEO_B, S_HL = S_TC + TC_B, S_HV = S_HL + HL_B;
  static constexpr uint32_t SLOT_B = S_HV + HV_B;
  static constexpr int HALO_FLOATS = (int)(S_HV / 4), SLOT_FLOATS = (int)(SLOT_B / 4);
  // shared-memory layout (bytes)
  static constexpr uint32_t OFF_BV = 0, OFF_BL = OFF_BV + 3 * BV_PART, OFF_SLOT = OFF_BL + 3 * BL_PART;
  static constexpr uint32_t OFF_BARY = OFF_SLOT + 2 * SLOT_B;
  // full[2], done[2], mvol, mlift, avol, alift, lst[2], hful[2]
  static constexpr uint32_t OFF_BARS = OFF_BARY + (uint32_t)NP * 3 * 8;
  static constexpr uint32_t OFF_MISC = OFF_BARS + 12 * 8;  // abort flag, TMEM base
  static constexpr uint32_t OFF_FMASK = (OFF_MISC + 16 + 15) & ~15u;
  static constexpr uint32_t OFF_FTAB = OFF_FMASK + ((NF + 15) & ~15);  // face-order rows of 16 bytes
  static constexpr uint32_t CONST_BYTES = 3 * BV_PART + 3 * BL_PART;  // the packed operand buffer
  // TMEM columns: acc_V, acc_L, then the three parts of the volume operand and of the LIFT operand (32
  // columns, 64 BF16 values of K, per part)
  static constexpr uint32_t T_ACCV = 0, T_ACCL = NV, T_AV = (uint32_t)((NV + NL + 31) & ~31), T_AL = T_AV + 3 * 32;
  static_assert(3 * NP <= 256 && NP <= 128 && NFP <= 16 && KV <= 64 && KL <= 64, "tile shapes");
  static_assert(T_AL + 3 * 32 <= (uint32_t)kTmCols, "TMEM columns");
  static_assert(HALO_FLOATS + kTmHalo * NFP <= 65536 && kTmTE * NP <= HALO_FLOATS, "16-bit slot positions");
};

template <int N>
__host__ __device__ constexpr uint32_t tm_smem(int ncodes) {
  return TmCfg<N>::OFF_FTAB + (uint32_t)ncodes * 16u;
}

// Round a pair to BF16 (one paired conversion): the packed bits, low half = x, and the residuals x - bf16(x).
__device__ __forceinline__ uint32_t bf16_pair(float &x, float &y) {
  const __nv_bfloat162 p = __float22bfloat162_rn(make_float2(x, y));
  const uint32_t w = *reinterpret_cast<const uint32_t *>(&p);
  x -= __uint_as_float(w << 16);
  y -= __uint_as_float(w & 0xffff0000u);
  return w;
}

// Split 8 consecutive K values of this thread's row into three BF16 parts and store part p's four packed
// columns at TMEM column `col + 32 p` of this warp's lanes.
__device__ __forceinline__ void tmem_split8(uint32_t col, const float (&v)[8]) {
  uint32_t w0[4], w1[4], w2[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float x = v[2 * q], y = v[2 * q + 1];  // residuals are exact in FP32
    w0[q] = bf16_pair(x, y);
    w1[q] = bf16_pair(x, y);
    w2[q] = bf16_pair(x, y);
  }
  tmem_st4(col, w0[0], w0[1], w0[2], w0[3]);
  tmem_st4(col + 32, w1[0], w1[1], w1[2], w1[3]);
  tmem_st4(col + 64, w2[0], w2[1], w2[2], w2[3]);
}

// 24 consecutive TMEM columns (three 8-column loads) of this warp's lanes under one wait.
__device__ __forceinline__ void tmem_ld24(uint32_t t0, float (&v)[24]) {
  uint32_t r[24];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%24];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%8,%9,%10,%11,%12,%13,%14,%15}, [%25];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%16,%17,%18,%19,%20,%21,%22,%23}, [%26];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23])
      : "r"(t0), "r"(t0 + 8), "r"(t0 + 16)
      : "memory");
#pragma unroll
  for (int j = 0; j < 24; ++j) v[j] = __uint_as_float(r[j]);
}

// (hn, ln) = (hi + lo) + b rn in error-free FP32 arithmetic, with b = bh + bl: the product by FMA residuals,
// the sums by Knuth's two-sum; about 47 significant bits, like an FP64 update rounded back to the pair.
__device__ __forceinline__ void stage_update(float hi, float lo, float rn, float bh, float bl, float &hn, float &ln) {
  const float p = bh * rn;
  const float ep = fmaf(bl, rn, fmaf(bh, rn, -p));  // b rn = p + ep
  const float s = hi + p;
  const float bb = s - hi;
  const float es = (hi - (s - bb)) + (p - bb);      // hi + p = s + es exactly
  const float t = lo + (ep + es);
  hn = s + t;
  const float bt = hn - s;
  ln = (s - (hn - bt)) + (t - bt);  // s + t = hn + ln exactly
}

// One GEMM of the split products: 6 MMAs per 16-wide K step into the accumulator at `acc`; A's three parts at
// TMEM columns a0, a0 + 32, a0 + 64 (8 columns per K step), B's in shared memory.
__device__ __forceinline__ void split_gemm(uint32_t acc, uint32_t a0, uint32_t b0, uint32_t b_part, int K, int NB,
                                           uint32_t idesc) {
  const int pa[6] = {0, 0, 1, 0, 2, 1}, pb[6] = {0, 1, 0, 2, 0, 1};
  for (int ks = 0; ks < K / 16; ++ks) {
    const uint32_t bo = (uint32_t)ks * 2 * (NB / 8) * 128;
#pragma unroll
    for (int t = 0; t < 6; ++t) {
      const uint64_t db = smem_desc(b0 + pb[t] * b_part + bo, (NB / 8) * 128, 128);
      tc_mma_ts(acc, a0 + 32u * pa[t] + 8u * ks, db, idesc, (ks > 0 || t > 0) ? 1u : 0u);
    }
  }
}

__device__ __forceinline__ int vload(const int *p) { return *reinterpret_cast<const volatile int *>(p); }

}  // namespace

// CW = 8 or 16 consumer warps: CW / 4 = 2 or 4 threads per element, each owning 4 / (CW / 4) faces.
// CONS: conservative form (w = u^2/2).
template <int N, int CW, bool CONS>
__global__ void __launch_bounds__(32 * (CW + 2), 1) rhs_stage_tcm_kernel(const MixedArgs A) {
  using C = TmCfg<N>;
  constexpr int TPE = CW / 4;  // threads per element
  constexpr int FPT = 4 / TPE; // faces per thread
  constexpr int KF = C::KF;
  static_assert(TPE == 2 || TPE == 4, "2 or 4 threads per element");
  constexpr bool cons = CONS;
  constexpr int NP = C::NP, NFP = C::NFP, NF = C::NF, KV = C::KV, KL = C::KL, NV = C::NV, NL = C::NL;
  constexpr int TE = kTmTE;
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char *sBV = sm + C::OFF_BV, *sBL = sm + C::OFF_BL;
  unsigned char *ring = sm + C::OFF_SLOT;
  double *sBary = reinterpret_cast<double *>(sm + C::OFF_BARY);
  // full: slot filled (the producer's bulk copies); done: slot finished (every consumer thread); mvol / mlift:
  // MMA group complete (tcgen05.commit); avol / alift: operand written into TMEM (every consumer thread); lst:
  // a slot's halo list arrived; hful: a slot's halo values arrived (every consumer thread's copies)
  uint64_t *full = reinterpret_cast<uint64_t *>(sm + C::OFF_BARS), *done = full + 2, *mvol = full + 4,
           *mlift = full + 5, *avol = full + 6, *alift = full + 7, *lst = full + 8, *hful = full + 10;
  int *sMisc = reinterpret_cast<int *>(sm + C::OFF_MISC);  // [0] abort flag, [1] TMEM base
  uint8_t *sFm = sm + C::OFF_FMASK, *sFt = sm + C::OFF_FTAB;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int G = gridDim.x;
  const int ncodes = A.ncodes;

  // constant operands, tables and barriers
  {
    const uint4 *src = reinterpret_cast<const uint4 *>(A.bmat);
    uint4 *dst = reinterpret_cast<uint4 *>(sBV);
    for (int x = tid; x < (int)(C::CONST_BYTES / 16); x += blockDim.x) dst[x] = src[x];
  }
  for (int x = tid; x < NP * 3; x += blockDim.x) sBary[x] = A.bary[x];
  for (int x = tid; x < NF; x += blockDim.x) sFm[x] = (uint8_t)A.fmask[x];
  for (int x = tid; x < ncodes * 16; x += blockDim.x) sFt[x] = (x & 15) < NFP ? A.ftab[(x >> 4) * NFP + (x & 15)] : 0;
  if (tid == 0) {
    for (int b = 0; b < 2; ++b) mbar_init(&full[b], 1);
    for (int b = 2; b < 4; ++b) mbar_init(&full[b], 32 * CW);
    mbar_init(mvol, 1);
    mbar_init(mlift, 1);
    mbar_init(avol, 32 * CW);
    mbar_init(alift, 32 * CW);
    mbar_init(&lst[0], 1);
    mbar_init(&lst[1], 1);
    mbar_init(&hful[0], 32 * CW);
    mbar_init(&hful[1], 32 * CW);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    sMisc[0] = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&sMisc[1])),
                 "r"(kTmCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_async_smem();  // the constant operands are read by the tensor cores (async proxy)
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = (uint32_t)sMisc[1];

  if (warp == CW + 1) {
    // producer warp, lane 0.  Slot s holds tile k, then k + 2.  Per tile: wait until every consumer thread has
    // finished tile k - 2 (done[s]), write its hi, lo and resu out with bulk stores (the ragged tail past the
    // last full 16 bytes was written by the consumers) and refill the slot once the stores have read it.  The
    // consumers read tile j's halo list while they work on tile j - 1 (tile 0's before their first tile), so
    // list j may replace list j - 2 once tile j - 3 is done: lists 0 and 1 go first, lists 2 and 3 after tile
    // 0 is done, list k + 1 after tile k - 2 is done.
    MTile held[2] = {};
    int kl[2] = {-1, -1}, kf[2] = {-1, -1};  // newest list request and newest fill of each slot
    auto store = [&](int s, const MTile &tl) {
      const uint32_t nbd = (((uint32_t)(tl.nelem * NP * 4)) & ~15u);
      unsigned char *slot = ring + (size_t)s * C::SLOT_B;
      if (nbd) {
        bulk_s2g(A.uhi_out + tl.node_base, slot, nbd);
        bulk_s2g(A.ulo_out + tl.node_base, slot + C::NODE_B, nbd);
        bulk_s2g(A.resu + tl.node_base, slot + 2 * C::NODE_B, nbd);
      }
      bulk_commit();
    };
    auto request_list = [&](int kk) {
      const int tt = blockIdx.x + kk * G;
      if (tt >= A.ntiles) return;
      const int h0 = A.halo_off[tt];
      const int nh = max(0, min(A.halo_off[tt + 1] - h0, kTmHalo));
      const uint32_t hb = (uint32_t)nh * 8u;  // even entry counts: a multiple of 16 bytes
      mbar_expect_tx(&lst[kk & 1], hb);
      if (hb) bulk_g2s(ring + (size_t)(kk & 1) * C::SLOT_B + C::S_HL, A.halo_list + 2 * (int64_t)h0, hb, &lst[kk & 1]);
      kl[kk & 1] = kk;
    };
    int k = 0;
    bool bad = false;
    for (;; ++k) {
      const int t = blockIdx.x + k * G;
      if (t >= A.ntiles) break;
      const int s = k & 1;
      unsigned char *slot = ring + (size_t)s * C::SLOT_B;
      const MTile tl = A.tiles[t];
      if (lane == 0) {
        if (k >= 2) {
          if (!mbar_wait_bounded(&done[s], (uint32_t)((k - 2) >> 1) & 1u, kSpinLimit)) {
            bad = true;
          } else {
            store(s, held[s]);
            bulk_wait_read_all();  // the slot may be refilled once the stores have read it
          }
        }
        if (!bad && vload(&sMisc[0])) bad = true;
        if (!bad) {
          if (k == 0 || k == 2) {
            request_list(k);
            request_list(k + 1);
          } else if (k >= 3) {
            request_list(k + 1);
          }
          held[s] = tl;
          const uint32_t nb = round16((uint32_t)(tl.nelem * NP * 4));
          const uint32_t gb = (uint32_t)tl.nelem * kMixedGeoWords * 4;
          const uint32_t cb = (uint32_t)tl.nelem * 16u;
          mbar_expect_tx(&full[s], 3 * nb + gb + cb);
          bulk_g2s(slot, A.uhi_in + tl.node_base, nb, &full[s]);
          bulk_g2s(slot + C::NODE_B, A.ulo_in + tl.node_base, nb, &full[s]);
          bulk_g2s(slot + 2 * C::NODE_B, A.resu + tl.node_base, nb, &full[s]);
          bulk_g2s(slot + C::S_GEO, A.geo + tl.elem_slot * kMixedGeoWords, gb, &full[s]);
          bulk_g2s(slot + C::S_TC, A.conn + tl.elem_slot * 4, cb, &full[s]);
          kf[s] = k;
        }
      }
      if (__shfl_sync(0xffffffffu, (int)bad, 0)) {
        bad = true;
        break;
      }
    }
    if (!bad && lane == 0) {
      // the last one or two tiles: write them back once their consumers are done
      for (int j = (k >= 2 ? k - 2 : 0); j < k && !bad; ++j) {
        if (!mbar_wait_bounded(&done[j & 1], (uint32_t)(j >> 1) & 1u, kSpinLimit)) {
          bad = true;
          break;
        }
        store(j & 1, held[j & 1]);
      }
      bulk_wait_read_all();
    }
    if (__shfl_sync(0xffffffffu, (int)bad, 0) || bad) {
      if (lane == 0) {
        atomicExch(A.status, kStatusTimeoutCode);
        *reinterpret_cast<volatile int *>(&sMisc[0]) = 1;
        // drain: the newest list request and fill of each slot must land before the CTA (and its smem) goes
        for (int s = 0; s < 2; ++s) {
          if (kl[s] >= 0) mbar_wait_bounded(&lst[s], (uint32_t)(kl[s] >> 1) & 1u, kSpinLimit);
          if (kf[s] >= 0) mbar_wait_bounded(&full[s], (uint32_t)(kf[s] >> 1) & 1u, kSpinLimit);
        }
        bulk_wait_read_all();
      }
    }
    return;
  }

  const uint32_t idv = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NV >> 3) << 17) | ((uint32_t)(TE >> 4) << 24);
  const uint32_t idl = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NL >> 3) << 17) | ((uint32_t)(TE >> 4) << 24);
  bool failed = false;
  if (warp == CW) {
    // MMA warp: once every consumer thread has written tile k's dw (avol), lane 0 issues the volume GEMM and
    // commits it to mvol; once they have written the flux (alift), the LIFT GEMM to mlift.
    int k = 0, kv = -1, kl = -1;  // last tiles whose volume / LIFT groups were committed
    for (;; ++k) {
      const int t = blockIdx.x + k * G;
      if (t >= A.ntiles) break;
      if (!mbar_wait_bounded(avol, (uint32_t)k & 1u, kSpinLimit) || vload(&sMisc[0])) {
        failed = true;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (lane == 0) {
        split_gemm(tmem + C::T_ACCV, tmem + C::T_AV, saddr(sBV), C::BV_PART, KV, NV, idv);
        tc_commit(mvol);
      }
      kv = k;
      __syncwarp();
      if (!mbar_wait_bounded(alift, (uint32_t)k & 1u, kSpinLimit) || vload(&sMisc[0])) {
        failed = true;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (lane == 0) {
        split_gemm(tmem + C::T_ACCL, tmem + C::T_AL, saddr(sBL), C::BL_PART, KL, NL, idl);
        tc_commit(mlift);
      }
      kl = k;
      __syncwarp();
    }
    if (failed) {
      if (lane == 0) {
        atomicExch(A.status, kStatusTimeoutCode);
        *reinterpret_cast<volatile int *>(&sMisc[0]) = 1;
      }
      // committed groups must complete before TMEM is freed (each wait is bounded)
      if (kv >= 0) mbar_wait_bounded(mvol, (uint32_t)kv & 1u, kSpinLimit);
      if (kl >= 0) mbar_wait_bounded(mlift, (uint32_t)kl & 1u, kSpinLimit);
    }
  } else {
    // consumers: thread (warp w, lane l) owns element e = 32 (w mod 4) + l and the share h = TPE - 1 - w / 4 of
    // its nodes (8-wide chunks h, h + TPE, ...) and faces (h FPT .. h FPT + FPT - 1)
    const int e = (warp & 3) * 32 + lane, h = TPE - 1 - (warp >> 2);
    const uint32_t lane_tmem = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    const float a = A.a, dt = A.dt;
    // b as an unevaluated pair of floats (b = bh + bl to about 2^-48) for the FP32 compensated update
    const float bh = __double2float_rn(A.b), bl = __double2float_rn(A.b - (double)bh);
    const int vA = A.vtx[0], vB = A.vtx[1], vC = A.vtx[2], vD = A.vtx[3];
    const uint32_t n_u32 = (uint32_t)min(A.n_u_values, (int64_t)0xffffffffu);
    // halo values of this CTA's tile kk into its slot: value v of the tile's halo (face v / NFP, point v mod
    // NFP, in the face's point order) is this thread's when v = tid mod 32 CW; every consumer thread arrives on
    // hful once its copies have landed
    auto gather_halo = [&](int kk) -> bool {
      const int tt = blockIdx.x + kk * G, ss = kk & 1;
      unsigned char *sl = ring + (size_t)ss * C::SLOT_B;
      const int h0 = A.halo_off[tt];
      const int nv = max(0, min(A.halo_off[tt + 1] - h0, kTmHalo)) * NFP;
      const bool ok = mbar_wait_bounded(&lst[ss], (uint32_t)(kk >> 1) & 1u, kSpinLimit);
      if (ok) {
        const int32_t *sL = reinterpret_cast<const int32_t *>(sl + C::S_HL);
        float *sHv = reinterpret_cast<float *>(sl + C::S_HV);
        bool gbad = false;
#pragma unroll 2
        for (int v = tid; v < nv; v += 32 * CW) {
          const int i = v / NFP, p = v - i * NFP;
          const int2 en = *reinterpret_cast<const int2 *>(sL + 2 * i);
          const uint32_t src = (uint32_t)en.x + sFt[min(max(en.y, 0), ncodes - 1) * 16 + p];
          if (src < n_u32)
            cp_async4(sHv + v, A.uhi_in + src);
          else
            gbad = true;
        }
        if (gbad) atomicExch(A.status, kStatusBadGather);
      }
      cp_async_arrive_noinc(&hful[ss]);  // always, so that the phase can complete
      return ok;
    };
    MTile tl_next{};
    if ((int)blockIdx.x < A.ntiles) {
      tl_next = A.tiles[blockIdx.x];
      if (!gather_halo(0)) failed = true;
    }
    int k = 0;
    for (; !failed; ++k) {
      const int t = blockIdx.x + k * G;
      if (t >= A.ntiles) break;
      const int s = k & 1;
      const MTile tl = tl_next;
      if (t + G < A.ntiles) tl_next = A.tiles[t + G];  // the next descriptor's load overlaps this tile
      const int ne = tl.nelem;
      const bool valid = e < ne;
      // the learned-sensor viscosity: this element's row of viscous right-hand side, if it has one (the load
      // is issued here so that its latency is spent before the epilogue)
      const int vrow = (A.vslot && valid) ? A.vslot[tl.elem_slot + e] : -1;
      const bool got = mbar_wait_bounded(&full[s], (uint32_t)(k >> 1) & 1u, kSpinLimit) &&
                       mbar_wait_bounded(&hful[s], (uint32_t)(k >> 1) & 1u, kSpinLimit);
      unsigned char *slot = ring + (size_t)s * C::SLOT_B;
      float *sHi = reinterpret_cast<float *>(slot);
      float *sLo = sHi + TE * NP;
      float *sRe = sLo + TE * NP;
      const float *sGeo = reinterpret_cast<const float *>(slot + C::S_GEO);
      const uint32_t *sTc = reinterpret_cast<const uint32_t *>(slot + C::S_TC);
      const int ee = valid ? e : 0;
      const float *hi = sHi + ee * NP;
      const float *lo = sLo + ee * NP;
      const float4 g0 = *reinterpret_cast<const float4 *>(sGeo + ee * kMixedGeoWords);
      const float4 g1 = *reinterpret_cast<const float4 *>(sGeo + ee * kMixedGeoWords + 4);
      const float cr = g0.x, cs = g0.y, ct = g0.z;
      const int64_t slot0 = tl.node_base;

      // ---- neighbour traces of this thread's faces: the slot position of each face's trace (inside the tile,
      // or the halo) and the face's point order ----
      float fl[FPT][KF];  // uP, then the flux; face h FPT + ff, point p
#pragma unroll
      for (int ff = 0; ff < FPT; ++ff) {
        const int f = h * FPT + ff;
        const uint32_t w = sTc[ee * 4 + f];
        const int off = (int)(w & 0xffffu);
        const int cd = min((int)((w >> 16) & 0xffu), ncodes - 1);
        const uint4 row = *reinterpret_cast<const uint4 *>(sFt + cd * 16);
        const uint32_t rw[4] = {row.x, row.y, row.z, row.w};
#pragma unroll
        for (int p = 0; p < KF; ++p) {
          float v = 0.f;
          if (p < NFP) v = sHi[min(off + (int)((rw[p >> 2] >> (8 * (p & 3))) & 0xffu), C::SLOT_FLOATS - 1)];
          fl[ff][p] = v;
        }
      }

      // ---- volume operand: dw = w - P1(w), this thread's 8-column chunks of K, split into TMEM ----
      const double uA = (double)hi[vA] + (double)lo[vA], uB = (double)hi[vB] + (double)lo[vB];
      const double uC = (double)hi[vC] + (double)lo[vC], uD = (double)hi[vD] + (double)lo[vD];
      const double wA = cons ? 0.5 * uA * uA : uA;
      const double dB = (cons ? 0.5 * uB * uB : uB) - wA;
      const double dC = (cons ? 0.5 * uC * uC : uC) - wA;
      const double dD = (cons ? 0.5 * uD * uD : uD) - wA;
      const float L0 = (float)(0.5 * ((double)cr * dB + (double)cs * dC + (double)ct * dD));
#pragma unroll
      for (int c = h; c < KV / 8; c += TPE) {
        float v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int j = 8 * c + q;
          v[q] = 0.f;
          if (j < NP) {
            const double uj = (double)hi[j] + (double)lo[j];
            const double wj = cons ? 0.5 * uj * uj : uj;
            v[q] = (float)((wj - wA) - (sBary[3 * j] * dB + sBary[3 * j + 1] * dC + sBary[3 * j + 2] * dD));
          }
        }
        tmem_split8(lane_tmem + C::T_AV + 4 * c, v);
      }
      tmem_wait_st();
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(avol);
      if (!got || vload(&sMisc[0])) {
        failed = true;
        break;
      }

      // ---- the Lax-Friedrichs flux 1/2 (uM-uP) (1/2 (uM+uP) g - max(|uM|,|uP|) |g|), into its own TMEM
      // columns while the volume MMAs run (the LIFT MMAs of the previous tile completed before its update) ----
#pragma unroll
      for (int ff = 0; ff < FPT; ++ff) {
        const int f = h * FPT + ff;
        const float g = f == 0 ? g0.w : f == 1 ? g1.x : f == 2 ? g1.y : g1.z, ga = fabsf(g);
        const uint8_t *fm = sFm + f * NFP;
#pragma unroll
        for (int p = 0; p < NFP; ++p) {
          const float uM = hi[fm[p]], uP = fl[ff][p];
          const float d = uM - uP;
          fl[ff][p] = 0.5f * d * (0.5f * (uM + uP) * g - fmaxf(fabsf(uM), fabsf(uP)) * ga);
        }
#pragma unroll
        for (int cq = 0; cq < KF / 8; ++cq) {
          float v[8];
#pragma unroll
          for (int q = 0; q < 8; ++q) v[q] = fl[ff][8 * cq + q];
          tmem_split8(lane_tmem + C::T_AL + (uint32_t)(f * KF + 8 * cq) / 2, v);
        }
      }
      tmem_wait_st();
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(alift);
      // the next tile's halo, while the MMAs run (its slot's previous halo was read before tile k - 1's LIFT)
      if (t + G < A.ntiles && !gather_halo(k + 1)) {
        failed = true;
        break;
      }

      // the viscous right-hand side of this thread's nodes, loaded while the MMAs run
      constexpr int NCE = ((NP + 7) / 8 + TPE - 1) / TPE;  // epilogue chunks per thread
      float vv[NCE][8];
#pragma unroll
      for (int cc = 0; cc < NCE; ++cc)
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int i = 8 * (h + TPE * cc) + q;
          vv[cc][q] = (vrow >= 0 && i < NP) ? (float)A.visc[(int64_t)vrow * NP + i] : 0.f;
        }

      // ---- volume epilogue while the LIFT MMAs run: t0 = a resu + dt vol for this thread's nodes ----
      const bool vdone = mbar_wait_bounded(mvol, (uint32_t)k & 1u, kSpinLimit);
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (!vdone) {
        failed = true;
        break;
      }
      float t0[NCE][8];
#pragma unroll
      for (int cc = 0; cc < NCE; ++cc) {
        const int c = h + TPE * cc;
        if (c < (NP + 7) / 8) {
          float dv[24];  // columns 3i+d of nodes 8c..8c+7
          tmem_ld24(lane_tmem + C::T_ACCV + 24 * c, dv);
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const int i = min(8 * c + q, NP - 1);
            const float dd = fmaf(cr, dv[3 * q], fmaf(cs, dv[3 * q + 1], fmaf(ct, dv[3 * q + 2], L0)));
            const float vol = cons ? -dd : -hi[i] * dd;
            t0[cc][q] = fmaf(a, sRe[ee * NP + i], dt * vol);
          }
        }
      }

      // ---- LIFT accumulator and the compensated stage update into the slot ----
      const bool ldone = mbar_wait_bounded(mlift, (uint32_t)k & 1u, kSpinLimit);
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t tail0 = ((uint32_t)(ne * NP * 4) & ~15u) / 4;  // nodes past the last full 16 B: plain stores
      if (ldone) {
#pragma unroll
        for (int cc = 0; cc < NCE; ++cc) {
          const int c = h + TPE * cc;
          if (c < (NP + 7) / 8) {
            float lf[8];
            tmem_ld8(lane_tmem + C::T_ACCL + 8 * c, lf);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              const int i = 8 * c + q;
              if (i < NP && valid) {
                const int o = e * NP + i;
                float rn = fmaf(dt, lf[q], t0[cc][q]);
                if (vrow >= 0) rn = fmaf(dt, vv[cc][q], rn);
                float hn, ln;
                stage_update(hi[i], lo[i], rn, bh, bl, hn, ln);
                sHi[o] = hn;
                sLo[o] = ln;
                sRe[o] = rn;
                if ((uint32_t)o >= tail0) {
                  A.uhi_out[slot0 + o] = hn;
                  A.ulo_out[slot0 + o] = ln;
                  A.resu[slot0 + o] = rn;
                }
              }
            }
          }
        }
      }
      if (!ldone) {
        failed = true;
        break;
      }
      fence_async_smem();  // the slot writes become visible to the producer's bulk stores
      mbar_arrive(&done[s]);
    }
    cp_async_wait_all();  // no halo copy may land after the CTA has gone
    if (failed && lane == 0) {
      atomicExch(A.status, kStatusTimeoutCode);
      *reinterpret_cast<volatile int *>(&sMisc[0]) = 1;
    }
  }  // consumers
  // consumers and the MMA warp: TMEM is freed once every access to it and every MMA into it is done
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  asm volatile("bar.sync 1, %0;" ::"n"(32 * (CW + 1)) : "memory");
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmCols));
}

namespace {

template <int N, int CW, bool CONS>
void tcm_attr() {
  static bool done[64] = {};
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev >= 0 && dev < 64 && done[dev]) return;
  cuda_check(cudaFuncSetAttribute(rhs_stage_tcm_kernel<N, CW, CONS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  227 * 1024),
             "tcm kernel smem attribute");
  if (dev >= 0 && dev < 64) done[dev] = true;
}

template <int N, int CW, bool CONS>
bool launch_tcm_n(const MixedArgs &A, int num_sms, cudaStream_t st, LaunchInfo *info) {
  // at least 116 KB of shared memory, so that one CTA (which holds all 512 TMEM columns) runs per SM
  const uint32_t smem = std::max<uint32_t>(tm_smem<N>(A.ncodes), 116u * 1024u);
  if (smem > 227u * 1024u) return false;
  tcm_attr<N, CW, CONS>();
  const int grid = std::max(1, std::min(num_sms, A.ntiles));
  rhs_stage_tcm_kernel<N, CW, CONS><<<grid, 32 * (CW + 2), smem, st>>>(A);
  cuda_check(cudaGetLastError(), "rhs_stage_tcm_kernel launch");
  if (info) *info = LaunchInfo{grid, 32 * (CW + 2), (int)smem, 1};
  return true;
}

template <int N>
void prepare_tcm_cw(int cw) {
  if (cw == 8) {
    tcm_attr<N, 8, false>();
    tcm_attr<N, 8, true>();
  } else if (cw == 16) {
    tcm_attr<N, 16, false>();
    tcm_attr<N, 16, true>();
  }
}

template <int N>
bool launch_tcm_cw(const MixedArgs &A, int cw, int num_sms, cudaStream_t st, LaunchInfo *info) {
  const bool cons = A.conservative != 0;
  if (cw == 8)
    return cons ? launch_tcm_n<N, 8, true>(A, num_sms, st, info) : launch_tcm_n<N, 8, false>(A, num_sms, st, info);
  if (cw == 16)
    return cons ? launch_tcm_n<N, 16, true>(A, num_sms, st, info) : launch_tcm_n<N, 16, false>(A, num_sms, st, info);
  return false;
}

template <int N>
void tcm_pack_n(const double *Dr, const double *Ds, const double *Dt, const double *LIFT, std::vector<uint16_t> &out) {
  using C = TmCfg<N>;
  constexpr int NP = C::NP, NF = C::NF, KV = C::KV, KL = C::KL, NV = C::NV, NL = C::NL;
  out.assign(C::CONST_BYTES / 2, 0);
  auto put = [&](size_t base, size_t part, int R, int r, int k, double x) {
    double rem = x;
    for (int p = 0; p < 3; ++p) {
      const __nv_bfloat16 v = __float2bfloat16_rn((float)rem);
      out[base + p * part + (size_t)kmaj(r, k, R)] = *reinterpret_cast<const uint16_t *>(&v);
      rem -= (double)__bfloat162float(v);
    }
  };
  const double *D[3] = {Dr, Ds, Dt};
  const size_t pv = (size_t)NV * KV, pl = (size_t)NL * KL;
  for (int i = 0; i < NP; ++i)
    for (int d = 0; d < 3; ++d)
      for (int j = 0; j < NP; ++j) put(0, pv, NV, 3 * i + d, j, D[d][i * NP + j]);
  constexpr int NFP = C::NFP, KF = C::KF;
  for (int i = 0; i < NP; ++i)
    for (int f = 0; f < 4; ++f)
      for (int q = 0; q < NFP; ++q) put(3 * pv, pl, NL, i, f * KF + q, LIFT[(size_t)i * NF + f * NFP + q]);
}

}  // namespace

int tcm_tile_elems() { return kTmTE; }

int tcm_halo_capacity() { return kTmHalo; }

int tcm_halo_floats(int N) {
  switch (N) {
    case 1: return TmCfg<1>::HALO_FLOATS;
    case 2: return TmCfg<2>::HALO_FLOATS;
    case 3: return TmCfg<3>::HALO_FLOATS;
    case 4: return TmCfg<4>::HALO_FLOATS;
    default: return 0;
  }
}

bool tcm_supported(int N) { return N >= 1 && N <= 4; }

void tcm_pack_operands(int N, const double *Dr, const double *Ds, const double *Dt, const double *LIFT,
                       std::vector<uint16_t> &out) {
  switch (N) {
    case 1: tcm_pack_n<1>(Dr, Ds, Dt, LIFT, out); break;
    case 2: tcm_pack_n<2>(Dr, Ds, Dt, LIFT, out); break;
    case 3: tcm_pack_n<3>(Dr, Ds, Dt, LIFT, out); break;
    case 4: tcm_pack_n<4>(Dr, Ds, Dt, LIFT, out); break;
    default: out.clear();
  }
}

void prepare_rhs_tcm(int N, int consumer_warps) {
  switch (N) {
    case 1: prepare_tcm_cw<1>(consumer_warps); break;
    case 2: prepare_tcm_cw<2>(consumer_warps); break;
    case 3: prepare_tcm_cw<3>(consumer_warps); break;
    case 4: prepare_tcm_cw<4>(consumer_warps); break;
    default: break;
  }
}

bool launch_rhs_tcm(int N, const MixedArgs &A, int consumer_warps, int num_sms, cudaStream_t st, LaunchInfo *info) {
  switch (N) {
    case 1: return launch_tcm_cw<1>(A, consumer_warps, num_sms, st, info);
    case 2: return launch_tcm_cw<2>(A, consumer_warps, num_sms, st, info);
    case 3: return launch_tcm_cw<3>(A, consumer_warps, num_sms, st, info);
    case 4: return launch_tcm_cw<4>(A, consumer_warps, num_sms, st, info);
    default: return false;
  }
}

}  // namespace dgk
