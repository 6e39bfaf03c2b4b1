// Precision form of the stage on the 5th-generation tensor cores (tcgen05, sm_100a): the volume and LIFT
// contractions as BF16 hi/lo split-operand GEMMs with FP32 accumulation in tensor memory (TMEM).
//
// Every operand x is split as x = hi + lo with hi = bf16(x), lo = bf16(x - hi), and a product as
// A B ~ A_hi B_hi + A_hi B_lo + A_lo B_hi (the lo*lo term, ~2^-16 of the product, is dropped), all three
// accumulated into one FP32 TMEM accumulator.  The state is the compensated FP32 pair of the mixed form
// (u = hi + lo), the residual FP32, the update FP64.  As in the mixed form the derivative operand is the field
// minus its linear vertex interpolant, whose exact derivative is added back, so the BF16 splitting error
// scales with the higher-order part of the field only.
//
// GEMM shapes per tile of TE = 64 elements (M = 128 matrix rows, rows past Np are zero):
//   acc_r/s/t[i][e] = sum_j D{r,s,t}[i][j] dw[e][j]      (K = Np rounded up to 16)
//   acc_L[i][e]     = sum_m LIFT[i][m] flux[e][m]         (K = 4 Nfp rounded up to 16)
// A operands (the constant matrices, hi and lo) are pre-arranged on the host in the K-major no-swizzle canonical
// layout (8 x 16-byte core matrices) and streamed per tile with 1-D bulk copies through a 2-slot ring; B
// operands (per-element dw and flux, hi and lo) are written by the threads into the same layout.  Thread t of
// the CTA (4 warps) owns matrix row / node t: it builds its node's B entries, and in the epilogue reads its
// TMEM lane (tcgen05.ld 32x32b) for the tile's elements and finishes dd, the volume term, the surface term and
// the compensated update.  One thread issues the MMAs (tcgen05.mma ... kind::f16) and the bulk copies; MMA
// completion is signalled through tcgen05.commit on mbarriers.  Every wait is bounded; TMEM is always freed.
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

constexpr int kTcTE = 64;    // elements per tile (the GEMM N)
constexpr int kTcM = 128;    // matrix rows per GEMM (the GEMM M)
constexpr int kTcCols = 256; // TMEM columns: 4 accumulators x 64

__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16 &h, __nv_bfloat16 &l) {
  h = __float2bfloat16_rn(x);
  l = __float2bfloat16_rn(x - __bfloat162float(h));
}

template <int N>
struct TcCfg {
  using O = Order<N>;
  static constexpr int NP = O::NP, NFP = O::NFP, NF = O::NF;
  static constexpr int KV = rup16(NP), KL = rup16(NF);
  static constexpr uint32_t AV_B = 2u * kTcM * KV * 2;  // one derivative matrix, hi then lo (bytes)
  static constexpr uint32_t AL_B = 2u * kTcM * KL * 2;  // LIFT, hi then lo
  static constexpr uint32_t ASLOT = AV_B > AL_B ? AV_B : AL_B;
  static constexpr uint32_t BV_B = 2u * kTcTE * KV * 2;  // dw hi then lo
  static constexpr uint32_t BL_B = 2u * kTcTE * KL * 2;  // flux hi then lo
  static constexpr uint32_t SMEM = 2 * ASLOT + BV_B + BL_B + kTcTE * 16 + 64;
  static_assert(NP <= kTcM, "the tensor-core form holds Np <= 128 rows");
};

}  // namespace

// A operands prepared by the host: for c = 0..3 (Dr, Ds, Dt, LIFT) the bytes at A + off[c], hi block then lo.
template <int N>
__global__ void __launch_bounds__(128, 1) rhs_stage_tc_kernel(const TcArgs A) {
  using C = TcCfg<N>;
  constexpr int NP = C::NP, NFP = C::NFP, NF = C::NF, KV = C::KV, KL = C::KL, TE = kTcTE;
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char *aslot[2] = {sm, sm + C::ASLOT};
  __nv_bfloat16 *bv = reinterpret_cast<__nv_bfloat16 *>(sm + 2 * C::ASLOT);             // [hi | lo]
  __nv_bfloat16 *bl = reinterpret_cast<__nv_bfloat16 *>(sm + 2 * C::ASLOT + C::BV_B);    // [hi | lo]
  float *sel = reinterpret_cast<float *>(sm + 2 * C::ASLOT + C::BV_B + C::BL_B);         // [TE][4] cr cs ct L0
  uint64_t *bars = reinterpret_cast<uint64_t *>(sel + TE * 4);  // full[2], mmadone[2], tiledone
  __shared__ uint32_t tmem_base;
  __shared__ int s_abort;
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t a_bytes[4] = {C::AV_B, C::AV_B, C::AV_B, C::AL_B};
  (void)NFP;

  // zero the B operands once: padded K columns and rows of partial tiles must read as zeros
  for (int x = tid; x < (int)((C::BV_B + C::BL_B) / 4); x += blockDim.x) reinterpret_cast<uint32_t *>(bv)[x] = 0u;
  if (tid == 0) {
    for (int b = 0; b < 5; ++b) mbar_init(&bars[b], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&tmem_base)),
                 "r"(kTcCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TE >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);

  // per-thread constants: node i = tid, its barycentric weights and the vertex nodes
  const int i = tid;
  const bool row = i < NP;
  double bw[3] = {0.0, 0.0, 0.0};
  if (row)
    for (int c = 0; c < 3; ++c) bw[c] = A.bary[3 * i + c];
  const int vA = A.vtx[0], vB = A.vtx[1], vC = A.vtx[2], vD = A.vtx[3];
  const int cons = A.conservative;
  const float a = A.a, dt = A.dt;
  const double b = A.b;

  uint32_t tiles_done = 0;  // completed phases of the tile barrier
  uint32_t full_phase[2] = {0, 0}, mma_phase[2] = {0, 0};
  bool pending[2] = {false, false};  // a bulk copy into the slot was issued and not yet waited for
  bool aborted = false;
  // thread 0 issues the A stream: load matrix c of every tile into slot (sequence index & 1)
  auto load_a = [&](int c, int slot) {
    mbar_expect_tx(&bars[slot], a_bytes[c]);
    bulk_g2s(aslot[slot], A.amat + A.aoff[c], a_bytes[c], &bars[slot]);
  };

  for (int t = blockIdx.x; t < A.ntiles; t += gridDim.x) {
    const MTile tl = A.tiles[t];
    const int ne = tl.nelem;
    // ---- B operands: dw = w - P1(w) (w = u or u^2/2) and the Lax-Friedrichs flux, split into BF16 hi/lo ----
    if (tid == 0) {  // start the A stream of this tile (slots are free: the previous tile's MMAs completed)
      load_a(0, 0);
      load_a(1, 1);
      pending[0] = pending[1] = true;
    }
    for (int e = 0; e < TE; ++e) {
      if (e >= ne) break;
      const int64_t nb = tl.node_base + (int64_t)e * NP;
      const float *hi = A.uhi_in + nb;
      const float *lo = A.ulo_in + nb;
      const double uA = (double)hi[vA] + (double)lo[vA], uB = (double)hi[vB] + (double)lo[vB];
      const double uC = (double)hi[vC] + (double)lo[vC], uD = (double)hi[vD] + (double)lo[vD];
      const double wA = cons ? 0.5 * uA * uA : uA;
      const double dB = (cons ? 0.5 * uB * uB : uB) - wA;
      const double dC = (cons ? 0.5 * uC * uC : uC) - wA;
      const double dD = (cons ? 0.5 * uD * uD : uD) - wA;
      if (row) {
        const double uj = (double)hi[i] + (double)lo[i];
        const double wj = cons ? 0.5 * uj * uj : uj;
        const float v = (float)((wj - wA) - (bw[0] * dB + bw[1] * dC + bw[2] * dD));
        __nv_bfloat16 h, l;
        split_bf16(v, h, l);
        const int o = kmaj(e, i, TE);
        bv[o] = h;
        bv[TE * KV + o] = l;
      }
      const float *ge = A.geo + (tl.elem_slot + e) * kMixedGeoWords;
      const int *ce = A.conn + (tl.elem_slot + e) * kMixedConnWords;
      if (tid == 0) {
        sel[e * 4 + 0] = ge[0];
        sel[e * 4 + 1] = ge[1];
        sel[e * 4 + 2] = ge[2];
        sel[e * 4 + 3] = (float)(0.5 * ((double)ge[0] * dB + (double)ge[1] * dC + (double)ge[2] * dD));
      }
      const uint32_t codes = (uint32_t)ce[4];
      for (int m = tid; m < NF; m += blockDim.x) {
        const int f = m / NFP, p = m - f * NFP;
        const int64_t base = ce[f];
        const int cd = min((int)((codes >> (8 * f)) & 0xffu), A.ncodes - 1);
        const int64_t idx = base + A.ftab[cd * NFP + p];
        const float uM = hi[A.fmask[m]];
        float uP;
        if ((uint64_t)idx < (uint64_t)A.n_u_values) {
          uP = A.uhi_in[idx];
        } else {
          uP = uM;
          atomicExch(A.status, kStatusBadGather);
        }
        const float g = ge[3 + f], ga = fabsf(g);
        const float d = uM - uP;
        const float fl = 0.5f * d * (0.5f * (uM + uP) * g - fmaxf(fabsf(uM), fabsf(uP)) * ga);
        __nv_bfloat16 h, l;
        split_bf16(fl, h, l);
        const int o = kmaj(e, m, TE);
        bl[o] = h;
        bl[TE * KL + o] = l;
      }
    }
    // partial tile: zero the rows of absent elements (they may hold the previous tile's values)
    if (ne < TE) {
      for (int x = tid; x < (TE - ne) * KV; x += blockDim.x) {
        const int e = ne + x / KV, k = x % KV, o = kmaj(e, k, TE);
        bv[o] = __float2bfloat16_rn(0.f);
        bv[TE * KV + o] = __float2bfloat16_rn(0.f);
      }
      for (int x = tid; x < (TE - ne) * KL; x += blockDim.x) {
        const int e = ne + x / KL, k = x % KL, o = kmaj(e, k, TE);
        bl[o] = __float2bfloat16_rn(0.f);
        bl[TE * KL + o] = __float2bfloat16_rn(0.f);
      }
    }
    fence_async_smem();
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    // ---- MMAs (one thread): Dr, Ds, Dt into accumulators 0..2, LIFT into accumulator 3 ----
    if (tid == 0) {
      bool ok = !s_abort;
      for (int c = 0; c < 4 && ok; ++c) {
        const int slot = c & 1;
        ok = mbar_wait_bounded(&bars[slot], full_phase[slot], kSpinLimit);
        if (!ok) break;
        full_phase[slot] ^= 1u;
        pending[slot] = false;
        const int K = c < 3 ? KV : KL;
        const uint32_t a0 = saddr(aslot[slot]), alo = a0 + (uint32_t)kTcM * K * 2;
        const uint32_t b0 = c < 3 ? saddr(bv) : saddr(bl);
        const uint32_t blo = b0 + (uint32_t)TE * K * 2;
        const uint32_t acc = tmem + (uint32_t)(c * TE);
        for (int ks = 0; ks < K / 16; ++ks) {
          const uint32_t ao = (uint32_t)ks * 2 * (kTcM / 8) * 128, bo = (uint32_t)ks * 2 * (TE / 8) * 128;
          const uint64_t dah = smem_desc(a0 + ao, (kTcM / 8) * 128, 128);
          const uint64_t dal = smem_desc(alo + ao, (kTcM / 8) * 128, 128);
          const uint64_t dbh = smem_desc(b0 + bo, (TE / 8) * 128, 128);
          const uint64_t dbl = smem_desc(blo + bo, (TE / 8) * 128, 128);
          tc_mma(acc, dah, dbh, idesc, ks > 0 ? 1u : 0u);
          tc_mma(acc, dah, dbl, idesc, 1u);
          tc_mma(acc, dal, dbh, idesc, 1u);
        }
        if (c < 2) {  // refill this slot with matrix c+2 once the MMAs reading it completed
          tc_commit(&bars[2 + slot]);
          ok = mbar_wait_bounded(&bars[2 + slot], mma_phase[slot], kSpinLimit);
          mma_phase[slot] ^= 1u;
          if (ok) {
            load_a(c + 2, slot);
            pending[slot] = true;
          }
        }
      }
      tc_commit(&bars[4]);  // completes once every MMA issued so far has completed
      if (!ok) {
        atomicExch(A.status, kStatusTimeoutCode);
        s_abort = 1;
      }
    }
    __syncthreads();
    // all threads: wait for the tile's MMAs (bounded, CTA-uniform decision)
    const bool done = mbar_wait_bounded(&bars[4], tiles_done & 1u, kSpinLimit);
    tiles_done++;
    if (!__syncthreads_and(done) || s_abort) {
      if (tid == 0) atomicExch(A.status, kStatusTimeoutCode);
      aborted = true;
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    // ---- epilogue: thread i reads TMEM lane i for the tile's elements ----
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < TE; c0 += 16) {
      float ur[16], us[16], ut[16], lf[16];
      tmem_ld16(lane_addr + c0, ur);
      tmem_ld16(lane_addr + TE + c0, us);
      tmem_ld16(lane_addr + 2 * TE + c0, ut);
      tmem_ld16(lane_addr + 3 * TE + c0, lf);
      if (!row) continue;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int e = c0 + j;
        if (e >= ne) break;
        const int64_t o = tl.node_base + (int64_t)e * NP + i;
        const float dd = fmaf(sel[e * 4 + 0], ur[j], fmaf(sel[e * 4 + 1], us[j], fmaf(sel[e * 4 + 2], ut[j], sel[e * 4 + 3])));
        const float h = A.uhi_in[o], l = A.ulo_in[o];
        const float vol = cons ? -dd : -h * dd;
        const float rn = fmaf(a, A.resu[o], dt * (vol + lf[j]));
        const double un = ((double)h + (double)l) + b * (double)rn;
        const float hn = __double2float_rn(un);
        A.uhi_out[o] = hn;
        A.ulo_out[o] = __double2float_rn(un - (double)hn);
        A.resu[o] = rn;
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();  // TMEM and the B operands are free for the next tile
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  // drain: no copy or MMA may be in flight when TMEM is freed and the CTA leaves
  if (tid == 0 && aborted) {
    for (int sl = 0; sl < 2; ++sl)
      if (pending[sl]) mbar_wait_bounded(&bars[sl], full_phase[sl], kSpinLimit);
    mbar_wait_bounded(&bars[4], tiles_done & 1u, kSpinLimit);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols));
}

namespace {

template <int N>
bool launch_tc_n(const TcArgs &A, int num_sms, cudaStream_t st, LaunchInfo *info) {
  using C = TcCfg<N>;
  static bool attr[64] = {};
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= 64 || !attr[dev]) {
    cuda_check(cudaFuncSetAttribute(rhs_stage_tc_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM),
               "tc kernel smem attribute");
    if (dev >= 0 && dev < 64) attr[dev] = true;
  }
  const int grid = std::max(1, std::min(num_sms, A.ntiles));
  rhs_stage_tc_kernel<N><<<grid, 128, C::SMEM, st>>>(A);
  cuda_check(cudaGetLastError(), "rhs_stage_tc_kernel launch");
  if (info) *info = LaunchInfo{grid, 128, (int)C::SMEM, 1};
  return true;
}

}  // namespace

int tc_tile_elems() { return kTcTE; }

// Host layout of the A operands: matrix c (rows x cols, row-major FP64) padded to 128 x rup16(cols), split into
// BF16 hi / lo and written K-major in 8 x 16-byte core matrices.  Returns the element offsets of the four
// matrices (hi block then lo block each).
void tc_pack_operands(const double *const *mats, const int *cols, int rows, std::vector<uint16_t> &out,
                      int64_t off[4]) {
  out.clear();
  for (int c = 0; c < 4; ++c) {
    const int K = rup16(cols[c]);
    off[c] = (int64_t)out.size() * 2;  // bytes
    std::vector<uint16_t> hi((size_t)kTcM * K, 0), lo((size_t)kTcM * K, 0);
    for (int r = 0; r < rows; ++r)
      for (int k = 0; k < cols[c]; ++k) {
        const float x = (float)mats[c][(size_t)r * cols[c] + k];
        const __nv_bfloat16 h = __float2bfloat16_rn(x);
        const __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
        hi[(size_t)kmaj(r, k, kTcM)] = *reinterpret_cast<const uint16_t *>(&h);
        lo[(size_t)kmaj(r, k, kTcM)] = *reinterpret_cast<const uint16_t *>(&l);
      }
    out.insert(out.end(), hi.begin(), hi.end());
    out.insert(out.end(), lo.begin(), lo.end());
  }
}

bool launch_rhs_tc(int N, const TcArgs &A, int num_sms, cudaStream_t st, LaunchInfo *info) {
  switch (N) {
    case 4: return launch_tc_n<4>(A, num_sms, st, info);
    case 5: return launch_tc_n<5>(A, num_sms, st, info);
    case 6: return launch_tc_n<6>(A, num_sms, st, info);
    case 7: return launch_tc_n<7>(A, num_sms, st, info);
    default: return false;
  }
}

}  // namespace dgk
