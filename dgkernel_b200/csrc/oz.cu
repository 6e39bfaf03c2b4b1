// Precision form of the mixed stage on the tensor cores with exact integer products (tcgen05 kind::i8, sm_100a),
// orders 4..7.
//
// The reference's warp & blend node set (element/library/gonudg/nodes3d.go:290-324) makes the high-order
// operators ill-conditioned: at order 7 max|Dr| = 9e4 and max|LIFT| = 1.9e5 with zero row sums, so a product
// with FP32-level rounding (2^-24 relative to sum |D_ij||u_j|) loses every digit of the derivative and the run
// leaves the stable range.  This kernel computes both element-local products to ~47 significant bits with the
// 8-bit integer tensor cores, in the manner of the Ozaki scheme (Ozaki, Ogita, Oishi and Rump, "Error-free
// transformations of matrix multiplication by using fast routines of matrix multiplication and its
// applications", Numerical Algorithms 59, 2012; on integer units: Uchino, Ozaki and Imamura, "Performance
// enhancement of the Ozaki scheme on integer matrix multiplication unit", IJHPCA 2025):
//
//   every row x of an operand is scaled by a power of two 2^E with |x| < 2^E, rounded once to the integer
//   n = rint(x 2^(B-E)) with B = 7 + 8 (S - 1) bits and cut into S digits, x ~ 2^(E-7) (d_0 + 2^-8 (d_1 + ...)),
//   d_0 = n >> (B - 7) in [-128, 127] (s8) and the bytes d_p in [0, 255] (u8) for p > 0 (exact integer shifts;
//   a floating-point remainder loop is not exact: for a tiny negative x, x - floor(x) rounds to 1); the digit
//   products d^A_p d^B_q with p + q = L summed over K are exact in
//   int32 (|sum| < 6 * 544 * 255^2 < 2^31), one TMEM accumulator per level L < S; the levels are joined in
//   FP64 by Horner's rule, h = acc_{S-1}; h = h 2^-8 + acc_L, and scaled by 2^(E_A + E_B - 14).
//   The operands carry B = 47 bits (S = 6) rounded to nearest, and the dropped terms p + q >= S stay below
//   about S 2^(-8S+2) of 2^(E_A+E_B) K.
//
// Orientation: the matrices are the MMA's A operand (M = 128 rows = output nodes, rows past Np zero) and the
// elements its B operand (N = 32 elements per tile), so TMEM lane i holds node i and column e element e, and
// one tile's 2 S accumulators (volume and LIFT per level, 32 columns each) fit the 512 TMEM columns.
//
//   volume: A_v[i][d KD + j] = D_d[i][j] (d = r, s, t; KD = rup32(Np)),  B_v[e][d KD + j] = c_d(e) dw_e(j)
//           (c_r = rx + ry + rz etc.: the Burgers flux uses the metrics only through these sums), so the
//           accumulator is dd = cr ur + cs us + ct ut directly;
//   LIFT:   A_l[i][m] = LIFT[i][m] (m = f Nfp + p),                      B_l[e][m] = flux_e(m).
//
// dw = w - P1(w) (w = u or u^2/2 minus its linear vertex interpolant, whose exact derivative L0 is added back),
// the Lax-Friedrichs flux and the digits are formed in FP64 from the compensated FP32 state (u = hi + lo); the
// stage update runs in FP64 and is rounded back to the (hi, lo) pair; the residual is FP32.
//
// The matrix digits (S x 128 rows x (3 KD + KL) bytes, a few hundred KB) do not fit shared memory: they are
// packed on the host in 4 KB chunks (one 32-wide K step of one digit) and streamed from L2 through a ring by a
// producer warp; every chunk of digit p feeds the S - p MMAs with element digits q <= S - 1 - p, which stay in
// shared memory for the tile.  CTA: 16 consumer warps (element digits, epilogue), one producer warp (state
// slots and matrix chunks, 1-D bulk copies), one MMA warp.  Every wait is bounded; a failed wait sets the
// status word, the CTA drains its copies and MMAs and frees TMEM.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "dg_kernels.cuh"
#include "kernels.hpp"
#include "runner.hpp"
#include "tcgen05.cuh"
#include "tma.cuh"

namespace dgk {

namespace {

constexpr int kOzTE = 32;         // elements per tile (the MMA's N; one compact-geometry slot)
constexpr int kOzCW = 16;         // consumer warps
constexpr int kOzRing = 16;       // matrix-chunk ring slots (64 KB in flight: covers the L2 latency)
constexpr int kOzSlots = 1;       // state slots: released after the digits are built, refilled during the MMAs
constexpr int kOzChunk = 4096;    // bytes of one matrix chunk: 128 rows x 32 K
constexpr int kOzTmemCols = 512;
constexpr int kOzDigits = 6;      // S: digits per operand (~47 significant bits)

__host__ __device__ constexpr int rup32(int x) { return (x + 31) & ~31; }

template <int N, int S>
struct OzCfg {
  using O = Order<N>;
  static constexpr int NP = O::NP, NFP = O::NFP, NF = O::NF;
  static constexpr int KD = rup32(NP), KV = 3 * KD, KL = rup32(NF), KT = KV + KL;
  static constexpr int CV = KV / 32, CT = KT / 32;       // 32-wide K chunks: volume, all
  static constexpr int XV = KD / 16, XL = KL / 16;       // 16-wide value groups: per volume direction, LIFT
  static constexpr int NX = XV + XL;                     // groups per element (a volume group feeds 3 directions)
  static constexpr int GPT = (NX + 15) / 16;             // groups per thread (16 threads per element)
  static constexpr uint32_t BCH = 1024;                  // bytes of one element-digit chunk: 32 rows x 32 K
  static constexpr uint32_t BSLICE = (uint32_t)CT * BCH; // one digit of the tile's element operand
  static constexpr uint32_t NODE_B = (uint32_t)kOzTE * NP * 4;
  static constexpr uint32_t SLOT_B = 2 * NODE_B + kOzTE * kMixedGeoWords * 4 + round16(kOzTE * kMixedConnWords * 4);
  // shared memory (bytes)
  static constexpr uint32_t OFF_B = 0;
  static constexpr uint32_t OFF_RING = OFF_B + S * BSLICE;
  static constexpr uint32_t OFF_SLOT = OFF_RING + kOzRing * kOzChunk;
  static constexpr uint32_t OFF_BARY = OFF_SLOT + kOzSlots * SLOT_B;
  static constexpr uint32_t OFF_L0 = OFF_BARY + NP * 3 * 8;               // double per element, 2 tile buffers
  static constexpr uint32_t OFF_EXP = OFF_L0 + 2 * kOzTE * 8;             // int: Ev[2][32], El[2][32], Fv[128], Fl[128]
  static constexpr uint32_t OFF_BARS = OFF_EXP + (4 * kOzTE + 2 * 128) * 4;
  // full[NS], sdone[NS], aful[R], aemp[R], bful, accf, tfree
  static constexpr int NBARS = 2 * kOzSlots + 2 * kOzRing + 3;
  static constexpr uint32_t OFF_MISC = OFF_BARS + NBARS * 8;              // abort flag, TMEM base
  static constexpr uint32_t OFF_PT = (OFF_MISC + 16 + 15) & ~15u;         // per face point: own node, face
  static constexpr uint32_t OFF_FTAB = OFF_PT + ((2 * NF + 15) & ~15);    // face-order rows of 64 bytes
  static_assert(NP <= 128 && NFP <= 64, "tile shapes");
  static_assert(S >= 2 && S <= 7, "digits");
};

template <int N, int S>
__host__ __device__ constexpr uint32_t oz_smem(int ncodes) {
  return OzCfg<N, S>::OFF_FTAB + (uint32_t)ncodes * 64u;
}

// 2^e as a double for |e| <= 1022 (built from the exponent field).
__device__ __forceinline__ double pow2(int e) {
  e = max(-1022, min(1023, e));
  return __longlong_as_double((long long)(e + 1023) << 52);
}

// Exponent E with |x| < 2^E for the largest |x| of a row (0 for an all-zero row): frexp's exponent.
__device__ __forceinline__ int row_exp(double amax) {
  if (!(amax > 0.0)) return -1100;  // all zero: every digit is zero whatever the scale
  int e;
  frexp(amax, &e);
  return e;
}

__device__ __forceinline__ void tc_mma_i8(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

// Digits of 16 values of a row with exponent E: each value rounded once to the integer n = rint(x 2^(B-E)),
// B = 7 + 8 (S - 1) (|n| <= 2^B; clamped to 2^B - 1 at the top), then cut by arithmetic shifts, which is exact:
// digit 0 = n >> (B - 7) in [-128, 127] (s8), digit p > 0 = the byte (n >> 8 (S - 1 - p)) & 255 (u8).  `scale`
// is 2^(B-E).  Digit p of value v goes to byte v of out[p].
template <int S>
__device__ __forceinline__ void digits16(const double (&x)[16], double scale, uint4 (&out)[S]) {
  constexpr int B = 7 + 8 * (S - 1);
  uint32_t w[S][4];
#pragma unroll
  for (int p = 0; p < S; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) w[p][q] = 0;
#pragma unroll
  for (int v = 0; v < 16; ++v) {
    long long n = __double2ll_rn(x[v] * scale);  // |x scale| < 2^B: exact scaling, one rounding
    n = min(n, (1ll << B) - 1);
#pragma unroll
    for (int p = 0; p < S; ++p)
      w[p][v >> 2] |= ((uint32_t)(n >> (8 * (S - 1 - p))) & 0xffu) << (8 * (v & 3));
  }
#pragma unroll
  for (int p = 0; p < S; ++p) out[p] = make_uint4(w[p][0], w[p][1], w[p][2], w[p][3]);
}

// 8 consecutive TMEM columns (int32) of this warp's 32 lanes starting at taddr; waits for the load.
__device__ __forceinline__ void tmem_ld8i(uint32_t taddr, int (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n\t"
               "tcgen05.wait::ld.sync.aligned;"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr)
               : "memory");
#pragma unroll
  for (int j = 0; j < 8; ++j) v[j] = (int)r[j];
}

// 8 consecutive TMEM columns (int32) of this warp's lanes, without waiting: complete with tmem_wait_ld().
__device__ __forceinline__ void tmem_ld8_nowait(uint32_t taddr, int (&v)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr)
               : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ int vload(const int *p) { return *reinterpret_cast<const volatile int *>(p); }

// Named barrier `id` over `n` threads that also ORs a predicate across them: every participant gets the same
// answer, so a decision taken on it (leave the tile loop) is uniform.
__device__ __forceinline__ bool bar_or(int id, int n, bool pred) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\tbar.red.or.pred p, %2, %3, q;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)pred), "r"(id), "r"(n)
      : "memory");
  return r != 0;
}

}  // namespace

template <int N, int S, bool CONS>
__global__ void __launch_bounds__(32 * (kOzCW + 2), 1) rhs_stage_oz_kernel(const OzArgs A) {
  using C = OzCfg<N, S>;
  constexpr int NP = C::NP, NFP = C::NFP, NF = C::NF, KD = C::KD, KV = C::KV, CV = C::CV, CT = C::CT;
  constexpr int XV = C::XV, NX = C::NX, GPT = C::GPT;
  constexpr int TE = kOzTE, NTH = 32 * kOzCW;
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char *sB = sm + C::OFF_B, *ring = sm + C::OFF_RING, *slots = sm + C::OFF_SLOT;
  double *sBary = reinterpret_cast<double *>(sm + C::OFF_BARY);
  double *sL02 = reinterpret_cast<double *>(sm + C::OFF_L0);
  // per-tile element exponents and L0, double-buffered by tile parity: tile k writes buffer k & 1 while the
  // epilogue of tile k - 1 may still read the other
  int *sEv2 = reinterpret_cast<int *>(sm + C::OFF_EXP), *sEl2 = sEv2 + 2 * TE, *sFv = sEl2 + 2 * TE, *sFl = sFv + 128;
  uint64_t *full = reinterpret_cast<uint64_t *>(sm + C::OFF_BARS), *sdone = full + kOzSlots, *aful = sdone + kOzSlots,
           *aemp = aful + kOzRing, *bful = aemp + kOzRing, *accf = bful + 1, *tfree = bful + 2;
  int *sMisc = reinterpret_cast<int *>(sm + C::OFF_MISC);  // [0] abort flag, [1] TMEM base
  uint8_t *sPt = sm + C::OFF_PT;                           // [m] own node of face point m, [NF + m] its face
  uint8_t *sFt = sm + C::OFF_FTAB;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int G = gridDim.x;

  for (int x = tid; x < NP * 3; x += blockDim.x) sBary[x] = A.bary[x];
  for (int x = tid; x < 128; x += blockDim.x) {
    sFv[x] = A.rexp[x];
    sFl[x] = A.rexp[128 + x];
  }
  for (int x = tid; x < NF; x += blockDim.x) {
    sPt[x] = (uint8_t)A.fmask[x];
    sPt[NF + x] = (uint8_t)(x / NFP);
  }
  for (int x = tid; x < A.ncodes * 64; x += blockDim.x)
    sFt[x] = (x & 63) < NFP ? A.ftab[(x >> 6) * NFP + (x & 63)] : 0;
  if (tid == 0) {
    for (int b = 0; b < kOzSlots; ++b) {
      mbar_init(&full[b], 1);
      mbar_init(&sdone[b], NTH);
    }
    for (int b = 0; b < kOzRing; ++b) {
      mbar_init(&aful[b], 1);
      mbar_init(&aemp[b], 1);
    }
    mbar_init(bful, NTH);
    mbar_init(accf, 1);
    mbar_init(tfree, NTH);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    sMisc[0] = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&sMisc[1])),
                 "r"(kOzTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = (uint32_t)sMisc[1];

  if (warp == kOzCW + 1) {
    // producer, lane 0: the state slots (two ahead at most) and the matrix chunks of every tile in order.  The
    // fill of tile k + 2 needs the epilogue of tile k to be done with its slot; it is issued as soon as that
    // shows, polled while waiting for ring slots, so that the matrix chunks of the next tile stream meanwhile.
    if (lane == 0) {
      bool bad = false;
      int nfill = 0;  // state fills issued (tiles 0 .. nfill - 1)
      int64_t g = 0;  // matrix chunks issued
      auto issue_fill = [&]() {
        const int k = nfill, s = k % kOzSlots;
        const MTile tl = A.tiles[blockIdx.x + k * G];
        unsigned char *slot = slots + (size_t)s * C::SLOT_B;
        const uint32_t nb = round16((uint32_t)(tl.nelem * NP * 4));
        const uint32_t gb = (uint32_t)tl.nelem * kMixedGeoWords * 4;
        const uint32_t cb = round16((uint32_t)(tl.nelem * kMixedConnWords * 4));
        mbar_expect_tx(&full[s], 2 * nb + gb + cb);
        bulk_g2s(slot, A.uhi_in + tl.node_base, nb, &full[s]);
        bulk_g2s(slot + C::NODE_B, A.ulo_in + tl.node_base, nb, &full[s]);
        bulk_g2s(slot + 2 * C::NODE_B, A.geo + tl.elem_slot * kMixedGeoWords, gb, &full[s]);
        bulk_g2s(slot + 2 * C::NODE_B + TE * kMixedGeoWords * 4, A.conn + tl.elem_slot * kMixedConnWords, cb,
                 &full[s]);
        ++nfill;
      };
      // issue the next fill if its tile exists and its slot is free (no wait)
      auto try_fill = [&]() {
        if (blockIdx.x + nfill * G >= A.ntiles) return;
        if (nfill >= kOzSlots &&
            !mbar_test_wait(&sdone[nfill % kOzSlots], (uint32_t)((nfill - kOzSlots) / kOzSlots) & 1u))
          return;
        issue_fill();
      };
      for (int i = 0; i < kOzSlots; ++i) try_fill();
      for (int k = 0; !bad; ++k) {
        const int t = blockIdx.x + k * G;
        if (t >= A.ntiles) break;
        for (int j = 0; j < S * CT; ++j, ++g) {
          const int rs = (int)(g % kOzRing);
          if (g >= kOzRing) {
            const uint32_t par = (uint32_t)((g / kOzRing) - 1) & 1u;
            uint32_t it = 0;
            while (!mbar_test_wait(&aemp[rs], par)) {
              try_fill();
              if (++it >= kSpinLimit) {
                bad = true;
                break;
              }
            }
          }
          if (bad || vload(&sMisc[0])) {
            bad = true;
            break;
          }
          mbar_expect_tx(&aful[rs], kOzChunk);
          bulk_g2s(ring + (size_t)rs * kOzChunk, A.amat + (size_t)j * kOzChunk, kOzChunk, &aful[rs]);
          try_fill();
        }
        // the fill of tile k + 1 must be out before the chunks of tile k + 1 can be used (bounded wait)
        if (!bad && blockIdx.x + (k + 1) * G < A.ntiles) {
          uint32_t it = 0;
          while (nfill < k + 2) {
            try_fill();
            if (++it >= kSpinLimit) {
              bad = true;
              break;
            }
          }
        }
      }
      if (bad) {
        atomicExch(A.status, kStatusTimeoutCode);
        *reinterpret_cast<volatile int *>(&sMisc[0]) = 1;
      }
      // drain: the newest fill of each state slot and of each ring slot must land before the CTA leaves
      for (int s = 0; s < kOzSlots && s < nfill; ++s) {
        const int kl = s + ((nfill - 1 - s) / kOzSlots) * kOzSlots;
        mbar_wait_bounded(&full[s], (uint32_t)(kl / kOzSlots) & 1u, kSpinLimit);
      }
      for (int64_t gl = g > kOzRing ? g - kOzRing : 0; gl < g; ++gl)
        mbar_wait_bounded(&aful[gl % kOzRing], (uint32_t)(gl / kOzRing) & 1u, kSpinLimit);
    }
    return;
  }

  bool failed = false;
  if (warp == kOzCW) {
    // MMA warp: tile k's element digits ready (bful) and tile k-1's accumulators read (tfree) -> for every
    // matrix chunk (p, c) from the ring, lane 0 issues the MMAs with element digits q <= S-1-p into level p + q
    constexpr uint32_t M = 128, NN = TE;
    const uint32_t idesc_base = (2u << 4) | ((NN >> 3) << 17) | ((M >> 4) << 24);  // S32 accumulate, K-major
    int64_t g = 0;
    int k = 0, kc = -1;
    for (;; ++k) {
      const int t = blockIdx.x + k * G;
      if (t >= A.ntiles) break;
      if (!mbar_wait_bounded(bful, (uint32_t)k & 1u, kSpinLimit) ||
          (k > 0 && !mbar_wait_bounded(tfree, (uint32_t)(k - 1) & 1u, kSpinLimit)) || vload(&sMisc[0])) {
        failed = true;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int p = 0; p < S && !failed; ++p) {
        for (int c = 0; c < CT; ++c, ++g) {
          const int rs = (int)(g % kOzRing);
          if (!mbar_wait_bounded(&aful[rs], (uint32_t)(g / kOzRing) & 1u, kSpinLimit)) {
            failed = true;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          if (lane == 0) {
            const uint64_t da = smem_desc(saddr(ring + (size_t)rs * kOzChunk), 2048, 128);
            const int acc = c < CV ? 0 : 1;
#pragma unroll
            for (int q = 0; q < S; ++q) {
              if (p + q < S) {
                const uint64_t db = smem_desc(saddr(sB + (size_t)q * C::BSLICE + (size_t)c * C::BCH), 512, 128);
                const uint32_t idesc = idesc_base | ((p == 0 ? 1u : 0u) << 7) | ((q == 0 ? 1u : 0u) << 10);
                const uint32_t col = (uint32_t)(((p + q) * 2 + acc) * TE);
                tc_mma_i8(tmem + col, da, db, idesc, (p == 0 && (c == 0 || c == CV)) ? 0u : 1u);
              }
            }
            tc_commit(&aemp[rs]);  // the ring slot is free once these MMAs have read it
          }
          __syncwarp();
        }
      }
      if (failed) break;
      if (lane == 0) tc_commit(accf);
      kc = k;
      __syncwarp();
    }
    if (failed) {
      if (lane == 0) {
        atomicExch(A.status, kStatusTimeoutCode);
        *reinterpret_cast<volatile int *>(&sMisc[0]) = 1;
      }
    }
    // every committed group completes before TMEM is freed (bounded)
    if (lane == 0 && g > 0) {
      const int64_t gl = g - 1;
      mbar_wait_bounded(&aemp[gl % kOzRing], (uint32_t)(gl / kOzRing) & 1u, kSpinLimit);
    }
    if (kc >= 0) mbar_wait_bounded(accf, (uint32_t)kc & 1u, kSpinLimit);
  } else {
    // consumers.  Element digits: thread (warp w, lane l) builds element e = 8 (w mod 4) + (l mod 8), value
    // groups x = 4 (w / 4) + l / 8 + 16 t (16 threads per element; a warp's 16-byte digit stores cover 8
    // elements x 4 groups, conflict-free).  Epilogue: warp w reads TMEM lane quarter w mod 4 (nodes
    // 32 (w mod 4) + l) for elements 8 (w / 4) .. 8 (w / 4) + 7.
    const int eb = (warp & 3) * 8 + (lane & 7), xg = (warp >> 2) * 4 + (lane >> 3);
    const int node = (warp & 3) * 32 + lane, e0 = (warp >> 2) * 8;
    const uint32_t lane_tmem = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    const double a = A.a, dt = A.dt, b = A.b;
    const int vA = A.vtx[0], vB = A.vtx[1], vC = A.vtx[2], vD = A.vtx[3];
    const int ncodes = A.ncodes;
    const uint32_t n_u32 = (uint32_t)min(A.n_u_values, (int64_t)0xffffffffu);
    MTile tl_next{};
    if ((int)blockIdx.x < A.ntiles) tl_next = A.tiles[blockIdx.x];
    bool pend = false;  // a wait of the previous tile failed: leave at the next barrier, together
    for (int k = 0;; ++k) {
      const int t = blockIdx.x + k * G;
      if (t >= A.ntiles) break;
      const int s = k % kOzSlots, tb = k & 1;  // state slot; tile-parity buffer of exponents and L0
      const MTile tl = tl_next;
      if (t + G < A.ntiles) tl_next = A.tiles[t + G];
      const int ne = tl.nelem;
      int *sEv = sEv2 + tb * TE, *sEl = sEl2 + tb * TE;
      double *sL0 = sL02 + tb * TE;
      if (tid < TE) {  // buffer s was last read by the epilogue of tile k - 2, finished before the last barrier
        sEv[tid] = -1100;
        sEl[tid] = -1100;
      }
      const bool got = mbar_wait_bounded(&full[s], (uint32_t)(k / kOzSlots) & 1u, kSpinLimit);
      if (bar_or(1, NTH, pend || !got || vload(&sMisc[0]) != 0)) {
        failed = true;
        break;
      }
      const float *sHi = reinterpret_cast<const float *>(slots + (size_t)s * C::SLOT_B);
      const float *sLo = sHi + TE * NP;
      const float *sGeo = sLo + TE * NP;
      const int *sCon = reinterpret_cast<const int *>(sGeo + TE * kMixedGeoWords);
      const int64_t slot0 = tl.node_base, slotn = (int64_t)ne * NP;

      // ---- element digits: values of this thread's groups, row maxima, digits ----
      const bool valid = eb < ne;
      const int ee = valid ? eb : 0;
      const float *hi = sHi + ee * NP;
      const float *lo = sLo + ee * NP;
      const float4 g0 = *reinterpret_cast<const float4 *>(sGeo + ee * kMixedGeoWords);
      const float4 g1 = *reinterpret_cast<const float4 *>(sGeo + ee * kMixedGeoWords + 4);
      const double cd[3] = {(double)g0.x, (double)g0.y, (double)g0.z};
      // element arithmetic in FP64 without contraction (dmul/dadd): every rounding is the restatement's, so the
      // digits, which feed an ill-conditioned product at high order, match it exactly
      const double uA = (double)hi[vA] + (double)lo[vA], uB = (double)hi[vB] + (double)lo[vB];
      const double uC = (double)hi[vC] + (double)lo[vC], uD = (double)hi[vD] + (double)lo[vD];
      const double wA = CONS ? __dmul_rn(0.5 * uA, uA) : uA;
      const double dB = (CONS ? __dmul_rn(0.5 * uB, uB) : uB) - wA;
      const double dC = (CONS ? __dmul_rn(0.5 * uC, uC) : uC) - wA;
      const double dD = (CONS ? __dmul_rn(0.5 * uD, uD) : uD) - wA;
      if (valid && xg == 0)
        sL0[eb] = 0.5 * __dadd_rn(__dadd_rn(__dmul_rn(cd[0], dB), __dmul_rn(cd[1], dC)), __dmul_rn(cd[2], dD));
      double val[GPT][16];
      double mv = 0.0, ml = 0.0;
      bool badg = false;
      const uint32_t codes = (uint32_t)sCon[ee * kMixedConnWords + 4];
#pragma unroll
      for (int gi = 0; gi < GPT; ++gi) {
        const int x = xg + 16 * gi;
#pragma unroll
        for (int v = 0; v < 16; ++v) val[gi][v] = 0.0;
        if (!valid || x >= NX) continue;
        if (x < XV) {  // dw at nodes 16 x .. 16 x + 15
#pragma unroll
          for (int v = 0; v < 16; ++v) {
            const int j = 16 * x + v;
            if (j < NP) {
              const double uj = (double)hi[j] + (double)lo[j];
              const double wj = CONS ? __dmul_rn(0.5 * uj, uj) : uj;
              const double lin = __dadd_rn(__dadd_rn(__dmul_rn(sBary[3 * j], dB), __dmul_rn(sBary[3 * j + 1], dC)),
                                           __dmul_rn(sBary[3 * j + 2], dD));
              const double dw = (wj - wA) - lin;
              val[gi][v] = dw;
              mv = fmax(mv, fabs(dw));
            }
          }
        } else {  // the Lax-Friedrichs flux at face points 16 (x - XV) ..: all gathers first, then the math
          float pH[16], pL[16];
#pragma unroll
          for (int v = 0; v < 16; ++v) {
            const int m = 16 * (x - XV) + v;
            pH[v] = 0.f;
            pL[v] = 0.f;
            if (m < NF) {
              const int f = sPt[NF + m], pp = m - f * NFP;
              const uint32_t nbs = (uint32_t)sCon[ee * kMixedConnWords + f];
              const int cdx = min((int)((codes >> (8 * f)) & 0xffu), ncodes - 1);
              const uint32_t idx = nbs + sFt[cdx * 64 + pp];
              if (idx < n_u32) {
                pH[v] = __ldg(A.uhi_in + idx);
                pL[v] = __ldg(A.ulo_in + idx);
              } else {  // out of range: reported, and the point takes its own trace (zero jump)
                badg = true;
                pH[v] = hi[sPt[m]];
                pL[v] = lo[sPt[m]];
              }
            }
          }
#pragma unroll
          for (int v = 0; v < 16; ++v) {
            const int m = 16 * (x - XV) + v;
            if (m < NF) {
              const int f = sPt[NF + m], own = sPt[m];
              const double uM = (double)hi[own] + (double)lo[own];
              const double uP = (double)pH[v] + (double)pL[v];
              const float gf = f == 0 ? g0.w : f == 1 ? g1.x : f == 2 ? g1.y : g1.z;
              const double gg = (double)gf, d = uM - uP;
              const double fl = __dmul_rn(0.5 * d, __dsub_rn(__dmul_rn(0.5 * (uM + uP), gg),
                                                            __dmul_rn(fmax(fabs(uM), fabs(uP)), fabs(gg))));
              val[gi][v] = fl;
              ml = fmax(ml, fabs(fl));
            }
          }
        }
      }
      if (badg) atomicExch(A.status, kStatusBadGather);
      if (valid) {
        const double cmax = fmax(fabs(cd[0]), fmax(fabs(cd[1]), fabs(cd[2])));
        if (mv > 0.0) atomicMax(&sEv[eb], row_exp(cmax * mv));
        if (ml > 0.0) atomicMax(&sEl[eb], row_exp(ml));
      }
      asm volatile("bar.sync 1, %0;" ::"n"(NTH) : "memory");
      if (valid) {
        constexpr int BITS = 7 + 8 * (S - 1);
        const double sv = pow2(BITS - sEv[eb]), sl = pow2(BITS - sEl[eb]);
#pragma unroll
        for (int gi = 0; gi < GPT; ++gi) {
          const int x = xg + 16 * gi;
          if (x >= NX) continue;
          if (x < XV) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              double y[16];
#pragma unroll
              for (int v = 0; v < 16; ++v) y[v] = cd[d] * val[gi][v];
              uint4 dg[S];
              digits16<S>(y, sv, dg);
              const int kk = d * KD + 16 * x;  // K index of the group's first value
              const uint32_t off = (uint32_t)(kk >> 5) * C::BCH + (uint32_t)(((kk >> 4) & 1) * 4 + (eb >> 3)) * 128 +
                                   (uint32_t)(eb & 7) * 16;
#pragma unroll
              for (int p = 0; p < S; ++p) *reinterpret_cast<uint4 *>(sB + (size_t)p * C::BSLICE + off) = dg[p];
            }
          } else {
            uint4 dg[S];
            digits16<S>(val[gi], sl, dg);
            const int kk = KV + 16 * (x - XV);
            const uint32_t off = (uint32_t)(kk >> 5) * C::BCH + (uint32_t)(((kk >> 4) & 1) * 4 + (eb >> 3)) * 128 +
                                 (uint32_t)(eb & 7) * 16;
#pragma unroll
            for (int p = 0; p < S; ++p) *reinterpret_cast<uint4 *>(sB + (size_t)p * C::BSLICE + off) = dg[p];
          }
        }
      }
      fence_async_smem();  // the digits are read by the tensor cores (async proxy)
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(bful);
      mbar_arrive(&sdone[s]);  // the state slot may be refilled (the epilogue reads the state from global)

      // ---- epilogue: join the levels, the stage update ----
      const bool done = mbar_wait_bounded(accf, (uint32_t)k & 1u, kSpinLimit);
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (!done) {
        pend = true;  // no TMEM reads; the others learn of it at the next barrier
        continue;
      }
      // this thread's state and residual first (coalesced over the lanes' nodes), then the accumulators
      float rs[8], hs[8], ls[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        rs[q] = hs[q] = ls[q] = 0.f;
        const int e = e0 + q;
        if (node < NP && e < ne) {
          const int64_t gi = slot0 + e * NP + node;
          rs[q] = A.resu[gi];
          hs[q] = __ldg(A.uhi_in + gi);
          ls[q] = __ldg(A.ulo_in + gi);
        }
      }
      // Horner over the levels, highest first, loading TMEM in batches of up to three levels per wait
      double hv[8], hl[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) hv[q] = hl[q] = 0.0;
#pragma unroll
      for (int acc = 0; acc < 2; ++acc) {
#pragma unroll
        for (int L0b = S - 1; L0b >= 0; L0b -= 3) {
          int av[3][8];
#pragma unroll
          for (int j = 0; j < 3; ++j)
            if (L0b - j >= 0) tmem_ld8_nowait(lane_tmem + (uint32_t)(((L0b - j) * 2 + acc) * TE + e0), av[j]);
          tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 3; ++j)
            if (L0b - j >= 0) {
#pragma unroll
              for (int q = 0; q < 8; ++q) {
                double &h = acc ? hl[q] : hv[q];
                h = fma(h, 0.00390625, (double)av[j][q]);
              }
            }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(tfree);  // the accumulators may be overwritten by the next tile's MMAs
      if (node < NP) {
        const int fv = sFv[node], flx = sFl[node];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int e = e0 + q;
          if (e < ne) {
            const double dd = __dadd_rn(__dmul_rn(hv[q], pow2(sEv[e] + fv - 14)), sL0[e]);
            const double lf = __dmul_rn(hl[q], pow2(sEl[e] + flx - 14));
            const double u = (double)hs[q] + (double)ls[q];
            const double rhs = __dadd_rn(CONS ? -dd : -__dmul_rn(u, dd), lf);
            const int64_t gi = slot0 + e * NP + node;
            const float rn = (float)__dadd_rn(__dmul_rn(a, (double)rs[q]), __dmul_rn(dt, rhs));
            const double un = __dadd_rn(u, __dmul_rn(b, (double)rn));
            const float hn = (float)un;
            A.uhi_out[gi] = hn;
            A.ulo_out[gi] = (float)(un - (double)hn);
            A.resu[gi] = rn;
          }
        }
      }
    }
    failed = failed || pend;
    if (failed && lane == 0) {
      atomicExch(A.status, kStatusTimeoutCode);
      *reinterpret_cast<volatile int *>(&sMisc[0]) = 1;
    }
  }
  // consumers and the MMA warp: TMEM is freed once every load from it and every MMA into it is done
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  asm volatile("bar.sync 2, %0;" ::"n"(32 * (kOzCW + 1)) : "memory");
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kOzTmemCols));
}

namespace {

template <int N, bool CONS>
void oz_attr() {
  static bool done[64] = {};
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev >= 0 && dev < 64 && done[dev]) return;
  cuda_check(cudaFuncSetAttribute(rhs_stage_oz_kernel<N, kOzDigits, CONS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  227 * 1024),
             "oz kernel smem attribute");
  if (dev >= 0 && dev < 64) done[dev] = true;
}

template <int N, bool CONS>
bool launch_oz_n(const OzArgs &A, int num_sms, cudaStream_t st, LaunchInfo *info) {
  // at least 116 KB so that one CTA holds an SM: each CTA allocates all 512 TMEM columns
  const uint32_t smem = std::max<uint32_t>(oz_smem<N, kOzDigits>(A.ncodes), 116u * 1024u);
  if (smem > 227u * 1024u) return false;
  oz_attr<N, CONS>();
  const int grid = std::max(1, std::min(num_sms, A.ntiles));
  rhs_stage_oz_kernel<N, kOzDigits, CONS><<<grid, 32 * (kOzCW + 2), smem, st>>>(A);
  cuda_check(cudaGetLastError(), "rhs_stage_oz_kernel launch");
  if (info) *info = LaunchInfo{grid, 32 * (kOzCW + 2), (int)smem, 1};
  return true;
}

// Digits of one row with exponent E, the same arithmetic as the kernel's digits16: n = rint(x 2^(B-E)),
// digit 0 = n >> (B - 7), digit p > 0 = the byte (n >> 8 (S - 1 - p)) & 255.
void row_digits(const double *x, int n, int E, int S, std::vector<std::vector<int>> &d) {
  const int B = 7 + 8 * (S - 1);
  d.assign((size_t)S, std::vector<int>((size_t)n, 0));
  const double scale = std::ldexp(1.0, B - E);
  for (int v = 0; v < n; ++v) {
    long long q = std::llrint(x[v] * scale);
    q = std::min(q, (1ll << B) - 1);
    d[0][(size_t)v] = (int)(q >> (B - 7));
    for (int p = 1; p < S; ++p) d[(size_t)p][(size_t)v] = (int)((q >> (8 * (S - 1 - p))) & 0xff);
  }
}

template <int N>
void oz_pack_n(const double *Dr, const double *Ds, const double *Dt, const double *LIFT, std::vector<uint8_t> &out,
               std::vector<int32_t> &rexp) {
  constexpr int S = kOzDigits;
  using C = OzCfg<N, S>;
  constexpr int NP = C::NP, NF = C::NF, KD = C::KD, KV = C::KV, KL = C::KL, CT = C::CT;
  out.assign((size_t)S * CT * kOzChunk, 0);
  rexp.assign(256, -1100);
  const double *D[3] = {Dr, Ds, Dt};
  std::vector<double> rv((size_t)KV), rl((size_t)KL);
  std::vector<std::vector<int>> dv, dl;
  for (int r = 0; r < 128; ++r) {
    std::fill(rv.begin(), rv.end(), 0.0);
    std::fill(rl.begin(), rl.end(), 0.0);
    if (r < NP) {
      for (int d = 0; d < 3; ++d)
        for (int j = 0; j < NP; ++j) rv[(size_t)(d * KD + j)] = D[d][(size_t)r * NP + j];
      for (int m = 0; m < NF; ++m) rl[(size_t)m] = LIFT[(size_t)r * NF + m];
    }
    double mv = 0.0, ml = 0.0;
    for (double v : rv) mv = std::max(mv, std::fabs(v));
    for (double v : rl) ml = std::max(ml, std::fabs(v));
    int ev = -1100, el = -1100;
    if (mv > 0.0) std::frexp(mv, &ev);
    if (ml > 0.0) std::frexp(ml, &el);
    rexp[(size_t)r] = ev;
    rexp[(size_t)(128 + r)] = el;
    row_digits(rv.data(), KV, mv > 0.0 ? ev : 0, S, dv);
    row_digits(rl.data(), KL, ml > 0.0 ? el : 0, S, dl);
    for (int p = 0; p < S; ++p)
      for (int k = 0; k < KV + KL; ++k) {
        const int c = k >> 5, kk = k & 31;
        const int v = k < KV ? dv[(size_t)p][(size_t)k] : dl[(size_t)p][(size_t)(k - KV)];
        const size_t off = (size_t)(p * CT + c) * kOzChunk + (size_t)(((kk >> 4) * 16 + (r >> 3)) * 128) +
                           (size_t)((r & 7) * 16 + (kk & 15));
        out[off] = (uint8_t)(v & 0xff);
      }
  }
}

}  // namespace

bool oz_supported(int N) { return N >= 4 && N <= 7; }
int oz_tile_elems() { return kOzTE; }
int oz_digits() { return kOzDigits; }

void oz_pack_operands(int N, const double *Dr, const double *Ds, const double *Dt, const double *LIFT,
                      std::vector<uint8_t> &digits, std::vector<int32_t> &rexp) {
  switch (N) {
    case 4: oz_pack_n<4>(Dr, Ds, Dt, LIFT, digits, rexp); break;
    case 5: oz_pack_n<5>(Dr, Ds, Dt, LIFT, digits, rexp); break;
    case 6: oz_pack_n<6>(Dr, Ds, Dt, LIFT, digits, rexp); break;
    case 7: oz_pack_n<7>(Dr, Ds, Dt, LIFT, digits, rexp); break;
    default: digits.clear(); rexp.clear();
  }
}

void prepare_rhs_oz(int N) {
  switch (N) {
    case 4: oz_attr<4, false>(); oz_attr<4, true>(); break;
    case 5: oz_attr<5, false>(); oz_attr<5, true>(); break;
    case 6: oz_attr<6, false>(); oz_attr<6, true>(); break;
    case 7: oz_attr<7, false>(); oz_attr<7, true>(); break;
    default: break;
  }
}

bool launch_rhs_oz(int N, const OzArgs &A, int conservative, int num_sms, cudaStream_t st, LaunchInfo *info) {
  const bool c = conservative != 0;
  switch (N) {
    case 4: return c ? launch_oz_n<4, true>(A, num_sms, st, info) : launch_oz_n<4, false>(A, num_sms, st, info);
    case 5: return c ? launch_oz_n<5, true>(A, num_sms, st, info) : launch_oz_n<5, false>(A, num_sms, st, info);
    case 6: return c ? launch_oz_n<6, true>(A, num_sms, st, info) : launch_oz_n<6, false>(A, num_sms, st, info);
    case 7: return c ? launch_oz_n<7, true>(A, num_sms, st, info) : launch_oz_n<7, false>(A, num_sms, st, info);
    default: return false;
  }
}

}  // namespace dgk
