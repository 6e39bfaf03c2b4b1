// Mixed-precision fused stage of the tet-DG right-hand side for sm_100a (operator "rhsStageMixed").
//
// Arithmetic.  The state is a compensated pair of FP32 arrays, u = hi + lo (about 48 significant bits), the
// LSERK residual is FP32, and the element-local products (Dr, Ds, Dt and LIFT) run in FP32 on the CUDA cores.
// Before differentiating, each element's linear interpolant through its four vertex nodes is subtracted in
// FP64 and its derivative (a difference of vertex values) is added back afterwards, so the FP32 products see
// only the small higher-order part of the field: the cancellation in D*u that limits a plain FP32 evaluation
// (row sums of D are zero, the entries are O(N^2)) no longer multiplies the rounding error.  The stage update
// u += b*resu runs in FP64 and is split back into hi and lo.
//
// Layout.  Straight-sided (affine) tetrahedra have constant metrics and constant face normals and Fscale, and
// the Burgers flux f(u) = (u^2/2)(1,1,1) uses them only through their (1,1,1) combinations: per element
// cr = rx+ry+rz, cs = sx+sy+sz, ct = tx+ty+tz, and per face g_f = Fscale_f (nx+ny+nz)_f.  These are 8 floats
// (32 B) per element instead of 9 metrics per node and 4 values per face point.  The gather map is compressed
// to one neighbour base per face (the value index of the neighbour element's first node) and a code per face
// that selects the node order of the neighbour's face points from a small table: 5 int32 (20 B) per element.
// Both compact forms are derived, when the operator is built, from the per-node arrays and the gather map, and
// are checked there to reproduce them exactly (connectivity) or to within 1e-6 relative (affinity).
//
// Execution.  One CTA per SM.  A producer warp streams 32-element slots (hi, lo, resu, geometry,
// connectivity) into a ring of shared-memory slots with 1-D bulk copies; each consumer warp owns one slot at a
// time with one element per lane.  Neighbour traces inside the slot are read from shared memory, the others
// from global memory (L2).  Results are written back into the slot and leave it with bulk stores.  Every wait
// on an mbarrier is bounded; a wait that gives up records kStatusTimeoutCode and the CTA drains and returns.
#include <algorithm>
#include <cstdint>

#include "dg_kernels.cuh"
#include "kernels.hpp"
#include "runner.hpp"
#include "tma.cuh"

namespace dgk {

template <int N>
struct MixedCfg {
  using O = Order<N>;
  static constexpr int NP = O::NP, NFP = O::NFP, NF = O::NF;
  static constexpr int TE = kMixedSlotElems;
  static constexpr int NPJ = (NP + 3) & ~3;  // derivative rows padded to whole float4 groups
  static constexpr uint32_t NODE_B = TE * NP * 4;
  static constexpr uint32_t GEO_B = TE * kMixedGeoWords * 4;
  static constexpr uint32_t CONN_B = TE * kMixedConnWords * 4;
  static constexpr uint32_t SLOT_B = 3 * NODE_B + GEO_B + CONN_B;  // hi, lo, resu, geometry, connectivity
  static constexpr uint32_t DM_FLOATS = NP * 3 * NPJ;             // [i][j/2][r,s,t][j%2] interleaved rows
  static constexpr uint32_t L_FLOATS = NP * NF;                   // LIFT rows
  static_assert(NODE_B % 16 == 0 && GEO_B % 16 == 0 && CONN_B % 16 == 0, "slot parts must stay 16-byte aligned");
  static_assert(NF % 4 == 0, "LIFT rows are read as float4");
};

// Shared-memory layout of the kernel (host and device agree through this function).
struct MixedSmem {
  uint32_t ring, dm, lift, bary, bars, tags, ftab, fmask, misc, total;
};
__host__ __device__ inline MixedSmem mixed_smem(uint32_t slot_b, uint32_t dm_floats, uint32_t l_floats, int np,
                                               int nfp, int ns, int ncodes) {
  MixedSmem m{};
  m.ring = 0;
  m.dm = m.ring + (uint32_t)ns * slot_b;
  m.lift = m.dm + dm_floats * 4;
  m.bary = m.lift + l_floats * 4;
  m.bars = m.bary + (uint32_t)np * 3 * 8;
  m.tags = m.bars + 2u * (uint32_t)ns * 8;
  m.ftab = m.tags + round16(4u * (uint32_t)ns);
  m.fmask = m.ftab + round16((uint32_t)(ncodes * nfp));
  m.misc = m.fmask + round16((uint32_t)(4 * nfp));
  m.total = m.misc + 32;
  return m;
}

namespace {

template <int N>
__device__ __forceinline__ void issue_slot(const MixedArgs &A, const MTile &tl, unsigned char *slot, uint64_t *bar) {
  using C = MixedCfg<N>;
  const uint32_t nb = round16((uint32_t)(tl.nelem * C::NP * 4));
  const uint32_t gb = (uint32_t)tl.nelem * kMixedGeoWords * 4;
  const uint32_t cb = round16((uint32_t)(tl.nelem * kMixedConnWords * 4));
  mbar_expect_tx(bar, 3 * nb + gb + cb);
  bulk_g2s(slot, A.uhi_in + tl.node_base, nb, bar);
  bulk_g2s(slot + C::NODE_B, A.ulo_in + tl.node_base, nb, bar);
  bulk_g2s(slot + 2 * C::NODE_B, A.resu + tl.node_base, nb, bar);
  bulk_g2s(slot + 3 * C::NODE_B, A.geo + tl.elem_slot * kMixedGeoWords, gb, bar);
  bulk_g2s(slot + 3 * C::NODE_B + C::GEO_B, A.conn + tl.elem_slot * kMixedConnWords, cb, bar);
}

__device__ __forceinline__ int vload(const int *p) { return *reinterpret_cast<const volatile int *>(p); }

}  // namespace

template <int N, int CW>
__global__ void __launch_bounds__(32 * (CW + 1), 1) rhs_stage_mixed_kernel(const MixedArgs A) {
  using C = MixedCfg<N>;
  constexpr int NP = C::NP, NFP = C::NFP, NF = C::NF, NPJ = C::NPJ, TE = C::TE;
  extern __shared__ __align__(128) unsigned char sm[];
  const int NS = A.ns;
  const MixedSmem L = mixed_smem(C::SLOT_B, C::DM_FLOATS, C::L_FLOATS, NP, NFP, NS, A.ncodes);
  unsigned char *ring = sm + L.ring;
  float *sDm = reinterpret_cast<float *>(sm + L.dm);
  float *sL = reinterpret_cast<float *>(sm + L.lift);
  double *sBary = reinterpret_cast<double *>(sm + L.bary);
  uint64_t *full = reinterpret_cast<uint64_t *>(sm + L.bars);
  uint64_t *empty = full + NS;
  uint8_t *sFt = sm + L.ftab;
  uint8_t *sFm = sm + L.fmask;
  int *sMisc = reinterpret_cast<int *>(sm + L.misc);  // [0..3] vertex nodes A..D, [4] abort flag
  int *sTag = reinterpret_cast<int *>(sm + L.tags);    // local tile index last issued into each slot
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int G = gridDim.x;

  for (int i = tid; i < (int)C::DM_FLOATS; i += blockDim.x) sDm[i] = A.Dm[i];
  for (int i = tid; i < (int)C::L_FLOATS; i += blockDim.x) sL[i] = A.lift[i];
  for (int i = tid; i < NP * 3; i += blockDim.x) sBary[i] = A.bary[i];
  for (int i = tid; i < A.ncodes * NFP; i += blockDim.x) sFt[i] = A.ftab[i];
  for (int i = tid; i < NF; i += blockDim.x) sFm[i] = (uint8_t)A.fmask[i];
  if (tid < 4) sMisc[tid] = A.vtx[tid];
  if (tid == 0) {
    sMisc[4] = 0;
    for (int s = 0; s < NS; ++s) {
      sTag[s] = -1;
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (warp == CW) {  // producer: lane 0 streams the slots of this CTA's tiles through the ring
    if (lane == 0) {
      int k = 0;
      bool bad = false;
      for (;; ++k) {
        const int t = blockIdx.x + k * G;
        if (t >= A.ntiles) break;
        const int s = k % NS;
        if (k >= NS && !mbar_wait_bounded(&empty[s], (uint32_t)((k / NS) - 1) & 1u, kSpinLimit)) {
          bad = true;
          break;
        }
        if (vload(&sMisc[4])) {
          bad = true;
          break;
        }
        *reinterpret_cast<volatile int *>(&sTag[s]) = k;  // fill k/NS of slot s is issued (k-NS was consumed)
        issue_slot<N>(A, A.tiles[t], ring + (size_t)s * C::SLOT_B, &full[s]);
      }
      if (bad) {
        atomicExch(A.status, kStatusTimeoutCode);
        *reinterpret_cast<volatile int *>(&sMisc[4]) = 1;
        // drain: the newest issued phase of every slot must land before the CTA (and its smem) goes away
        for (int s = 0; s < NS && s < k; ++s) {
          const int kl = s + ((k - 1 - s) / NS) * NS;
          mbar_wait_bounded(&full[s], (uint32_t)(kl / NS) & 1u, kSpinLimit);
        }
      }
    }
    return;
  }

  const float a = A.a, dt = A.dt;
  const double b = A.b;
  const int cons = A.conservative;
  const int vA = sMisc[0], vB = sMisc[1], vC = sMisc[2], vD = sMisc[3];
  const int ncodes = A.ncodes;
  for (int k = warp;; k += CW) {
    const int t = blockIdx.x + k * G;
    if (t >= A.ntiles) break;
    const int s = k % NS;
    // Warps own fixed tiles but share the ring, so a warp can reach tile k while the slot still waits for an
    // earlier occupant; its parity wait is unambiguous only once the fill before k's has completed, which the
    // producer guarantees by the time it tags the slot with k.
    bool ok = false;
    for (uint32_t it = 0; it < kSpinLimit; ++it)
      if (vload(&sTag[s]) == k || vload(&sMisc[4])) {
        ok = vload(&sTag[s]) == k;
        break;
      }
    ok = ok && mbar_wait_bounded(&full[s], (uint32_t)(k / NS) & 1u, kSpinLimit);
    ok = __all_sync(0xffffffffu, ok) && !vload(&sMisc[4]);
    if (!ok) {
      if (lane == 0) {
        atomicExch(A.status, kStatusTimeoutCode);
        *reinterpret_cast<volatile int *>(&sMisc[4]) = 1;
      }
      break;
    }
    const MTile tl = A.tiles[t];
    const int ne = tl.nelem;
    const bool valid = lane < ne;
    const int e = valid ? lane : 0;  // idle lanes mirror element 0 and store nothing
    float *sHi = reinterpret_cast<float *>(ring + (size_t)s * C::SLOT_B);
    float *sLo = sHi + TE * NP;
    float *sRe = sLo + TE * NP;
    const float *sGeo = sRe + TE * NP;
    const int *sCon = reinterpret_cast<const int *>(sGeo + TE * kMixedGeoWords);
    const float *hi = sHi + e * NP;
    const float *lo = sLo + e * NP;
    const float4 g0 = *reinterpret_cast<const float4 *>(sGeo + e * kMixedGeoWords);
    const float4 g1 = *reinterpret_cast<const float4 *>(sGeo + e * kMixedGeoWords + 4);
    const float cr = g0.x, cs = g0.y, ct = g0.z;
    const float gf[4] = {g0.w, g1.x, g1.y, g1.z};
    const uint32_t codes = (uint32_t)sCon[e * kMixedConnWords + 4];
    const int64_t slot0 = tl.node_base, slotn = (int64_t)ne * NP;

    // field minus its linear interpolant through the vertex nodes (FP64), w = u or u^2/2; pairs of columns
    const double uA = (double)hi[vA] + (double)lo[vA], uB = (double)hi[vB] + (double)lo[vB];
    const double uC = (double)hi[vC] + (double)lo[vC], uD = (double)hi[vD] + (double)lo[vD];
    const double wA = cons ? 0.5 * uA * uA : uA;
    const double dB = (cons ? 0.5 * uB * uB : uB) - wA;
    const double dC = (cons ? 0.5 * uC * uC : uC) - wA;
    const double dD = (cons ? 0.5 * uD * uD : uD) - wA;
    float2 du[NPJ / 2];
#pragma unroll
    for (int j = 0; j < NPJ; ++j) {
      float v = 0.f;
      if (j < NP) {
        const double uj = (double)hi[j] + (double)lo[j];
        const double wj = cons ? 0.5 * uj * uj : uj;
        v = (float)((wj - wA) - (sBary[3 * j] * dB + sBary[3 * j + 1] * dC + sBary[3 * j + 2] * dD));
      }
      if (j & 1)
        du[j / 2].y = v;
      else
        du[j / 2].x = v;
    }
    // derivative of the linear part along (1,1,1): d/dr = (wB-wA)/2 and likewise for s, t
    const float L0 = (float)(0.5 * ((double)cr * dB + (double)cs * dC + (double)ct * dD));

    // Volume pass: dd_i = cr (Dr dw)_i + cs (Ds dw)_i + ct (Dt dw)_i + L0 with paired FMAs; the residual slot
    // receives a*resu + dt*vol (the surface term is added in the next pass).
#pragma unroll 1
    for (int i = 0; i < NP; ++i) {
      const float4 *Dq = reinterpret_cast<const float4 *>(sDm + i * 3 * NPJ);
      float2 ar = make_float2(0.f, 0.f), as = ar, at = ar, br = ar, bs = ar, bt = ar;
#pragma unroll
      for (int g = 0; g < NPJ / 4; ++g) {
        const float4 q0 = Dq[3 * g], q1 = Dq[3 * g + 1], q2 = Dq[3 * g + 2];
        ar = __ffma2_rn(make_float2(q0.x, q0.y), du[2 * g], ar);
        as = __ffma2_rn(make_float2(q0.z, q0.w), du[2 * g], as);
        at = __ffma2_rn(make_float2(q1.x, q1.y), du[2 * g], at);
        br = __ffma2_rn(make_float2(q1.z, q1.w), du[2 * g + 1], br);
        bs = __ffma2_rn(make_float2(q2.x, q2.y), du[2 * g + 1], bs);
        bt = __ffma2_rn(make_float2(q2.z, q2.w), du[2 * g + 1], bt);
      }
      const float ur = (ar.x + ar.y) + (br.x + br.y);
      const float us = (as.x + as.y) + (bs.x + bs.y);
      const float ut = (at.x + at.y) + (bt.x + bt.y);
      const float dd = fmaf(cr, ur, fmaf(cs, us, fmaf(ct, ut, L0)));
      const float vol = cons ? -dd : -hi[i] * dd;
      const int o = e * NP + i;
      const float t0 = fmaf(a, sRe[o], dt * vol);
      if (valid) sRe[o] = t0;
    }

    // Neighbour traces uP: inside the slot from shared memory, otherwise from the previous stage's state, read
    // through one generic address per point (no divergent branch between the two memories).  They are loaded
    // after the volume pass so that the pass runs with the fewest live registers.
    float fl[NF];
    bool bad = false;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      const int64_t nb = sCon[e * kMixedConnWords + f];
      const int cd = min((int)((codes >> (8 * f)) & 0xffu), ncodes - 1);
      const uint8_t *ft = sFt + cd * NFP;
      const bool ins = (uint64_t)(nb - slot0) < (uint64_t)slotn;
#pragma unroll
      for (int i = 0; i < NFP; ++i) {
        const int64_t idx = nb + ft[i];
        const bool okg = (uint64_t)idx < (uint64_t)A.n_u_values;
        bad |= valid && !ins && !okg;
        const float *src = ins ? sHi + (idx - slot0) : (okg ? A.uhi_in + idx : hi + sFm[f * NFP + i]);
        fl[f * NFP + i] = *src;
      }
    }
    if (bad) atomicExch(A.status, kStatusBadGather);
    // Lax-Friedrichs surface term times Fscale: 1/2 (uM-uP) (1/2 (uM+uP) g - max(|uM|,|uP|) |g|)
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      const float g = gf[f], ga = fabsf(g);
#pragma unroll
      for (int i = 0; i < NFP; ++i) {
        const float uM = hi[sFm[f * NFP + i]];
        const float uP = fl[f * NFP + i];
        const float d = uM - uP;
        fl[f * NFP + i] = 0.5f * d * (0.5f * (uM + uP) * g - fmaxf(fabsf(uM), fabsf(uP)) * ga);
      }
    }
    __syncwarp();  // every lane has read the slot's traces before any lane overwrites its own state

    // Surface pass: LIFT row times the flux (paired FMAs), then the stage update in FP64, split into hi + lo.
    const uint32_t tail0 = ((uint32_t)(ne * NP * 4) & ~15u) / 4;  // nodes past the last full 16 B: plain stores
#pragma unroll 1
    for (int i = 0; i < NP; ++i) {
      const float4 *Lq = reinterpret_cast<const float4 *>(sL + i * NF);
      float2 l0 = make_float2(0.f, 0.f), l1 = l0, l2 = l0, l3 = l0;
#pragma unroll
      for (int g = 0; g < NF / 4; ++g) {
        const float4 m = Lq[g];
        if (g & 1) {
          l2 = __ffma2_rn(make_float2(m.x, m.y), make_float2(fl[4 * g], fl[4 * g + 1]), l2);
          l3 = __ffma2_rn(make_float2(m.z, m.w), make_float2(fl[4 * g + 2], fl[4 * g + 3]), l3);
        } else {
          l0 = __ffma2_rn(make_float2(m.x, m.y), make_float2(fl[4 * g], fl[4 * g + 1]), l0);
          l1 = __ffma2_rn(make_float2(m.z, m.w), make_float2(fl[4 * g + 2], fl[4 * g + 3]), l1);
        }
      }
      const float lift = ((l0.x + l0.y) + (l1.x + l1.y)) + ((l2.x + l2.y) + (l3.x + l3.y));
      const int o = e * NP + i;
      const float rn = fmaf(dt, lift, sRe[o]);
      const double un = ((double)hi[i] + (double)lo[i]) + b * (double)rn;
      const float hn = __double2float_rn(un);
      const float ln = __double2float_rn(un - (double)hn);
      if (valid) {
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
    fence_async_smem();  // this lane's slot writes become visible to the bulk stores
    __syncwarp();
    if (lane == 0) {
      const uint32_t nbd = tail0 * 4;
      if (nbd) {
        bulk_s2g(A.uhi_out + slot0, sHi, nbd);
        bulk_s2g(A.ulo_out + slot0, sLo, nbd);
        bulk_s2g(A.resu + slot0, sRe, nbd);
      }
      bulk_commit();
      bulk_wait_read_all();  // the slot may be refilled once the stores have read it
      mbar_arrive(&empty[s]);
    }
    __syncwarp();
  }
}

namespace {

constexpr uint32_t kSmemBudget = 227 * 1024;

// The shared-memory opt-in of one instantiation, raised to the budget once per device (so that launches recorded
// by a stream capture need no attribute call).
template <int N, int CW>
void mixed_attr() {
  static bool done[64] = {};
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev >= 0 && dev < 64 && done[dev]) return;
  cuda_check(cudaFuncSetAttribute(rhs_stage_mixed_kernel<N, CW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kSmemBudget),
             "mixed kernel smem attribute");
  if (dev >= 0 && dev < 64) done[dev] = true;
}

template <int N, int CW>
bool launch_mixed_n(const MixedArgs &A0, int ring_max, int num_sms, cudaStream_t st, LaunchInfo *info) {
  using C = MixedCfg<N>;
  MixedArgs A = A0;
  int ns = 0;
  const int cap = ring_max > 0 ? std::min(ring_max, 24) : 24;
  while (ns < cap && mixed_smem(C::SLOT_B, C::DM_FLOATS, C::L_FLOATS, C::NP, C::NFP, ns + 1, A.ncodes).total <=
                         kSmemBudget)
    ++ns;
  if (ns < 2) return false;
  A.ns = ns;
  const uint32_t smem = mixed_smem(C::SLOT_B, C::DM_FLOATS, C::L_FLOATS, C::NP, C::NFP, ns, A.ncodes).total;
  auto kern = rhs_stage_mixed_kernel<N, CW>;
  mixed_attr<N, CW>();
  const int grid = std::max(1, std::min(num_sms, A.ntiles));
  kern<<<grid, 32 * (CW + 1), smem, st>>>(A);
  cuda_check(cudaGetLastError(), "rhs_stage_mixed_kernel launch");
  if (info) *info = LaunchInfo{grid, 32 * (CW + 1), (int)smem, 1};
  return true;
}

template <int N>
void prepare_mixed_cw(int cw) {
  if (cw == 4) mixed_attr<N, 4>();
  if (cw == 8) mixed_attr<N, 8>();
  if (cw == 11) mixed_attr<N, 11>();
}

template <int N>
bool launch_mixed_cw(const MixedArgs &A, int cw, int ring_max, int num_sms, cudaStream_t st, LaunchInfo *info) {
  switch (cw) {
    case 4: return launch_mixed_n<N, 4>(A, ring_max, num_sms, st, info);
    case 8: return launch_mixed_n<N, 8>(A, ring_max, num_sms, st, info);
    case 11: return launch_mixed_n<N, 11>(A, ring_max, num_sms, st, info);
    default: return false;
  }
}

// Compact per-element geometry: cr, cs, ct and g_f = Fscale_f (nx+ny+nz)_f, with an affinity check (1e-6
// relative: node-to-node roundoff of the FP64 metrics reaches ~1e-9 at order 7, a curved element differs by O(h)).
template <typename T>
__global__ void compact_geometry_kernel(CompactGeoArgs<T> g) {
  const int64_t total = g.elem_total;
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < total; x += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = g.npart - 1;  // partition holding global element x
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      if (g.elem_prefix[mid] <= x) lo = mid; else hi = mid - 1;
    }
    const int p = lo;
    const int64_t e = x - g.elem_prefix[p];
    const int64_t slot = g.slot_prefix[p] + e;
    const int64_t nb = g.node_off[p] + e * g.np;
    const int64_t fb = g.face_off[p] + e * g.nf;
    double c[3], scale = 0.0;
    for (int d = 0; d < 3; ++d) {
      c[d] = (double)g.geo[3 * d][nb] + (double)g.geo[3 * d + 1][nb] + (double)g.geo[3 * d + 2][nb];
      for (int q = 0; q < 3; ++q) scale = fmax(scale, fabs((double)g.geo[3 * d + q][nb]));
    }
    bool bad = false;
    for (int n = 1; n < g.np; ++n)
      for (int d = 0; d < 3; ++d) {
        const double v = (double)g.geo[3 * d][nb + n] + (double)g.geo[3 * d + 1][nb + n] +
                         (double)g.geo[3 * d + 2][nb + n];
        bad = bad || !(fabs(v - c[d]) <= 1e-6 * scale);
      }
    const int nfp = g.nf / 4;
    double gf[4];
    for (int f = 0; f < 4; ++f) {
      const int64_t q0 = fb + f * nfp;
      gf[f] = (double)g.face[3][q0] * ((double)g.face[0][q0] + (double)g.face[1][q0] + (double)g.face[2][q0]);
      const double fs = fabs((double)g.face[3][q0]) *
                        (fabs((double)g.face[0][q0]) + fabs((double)g.face[1][q0]) + fabs((double)g.face[2][q0]));
      for (int i = 1; i < nfp; ++i) {
        const int64_t q = q0 + i;
        const double v = (double)g.face[3][q] * ((double)g.face[0][q] + (double)g.face[1][q] + (double)g.face[2][q]);
        bad = bad || !(fabs(v - gf[f]) <= 1e-6 * fs);
      }
    }
    float *o = g.out + slot * kMixedGeoWords;
    o[0] = (float)c[0];
    o[1] = (float)c[1];
    o[2] = (float)c[2];
    for (int f = 0; f < 4; ++f) o[3 + f] = (float)gf[f];
    o[7] = 0.f;
    if (bad) atomicAdd(g.bad, 1);
  }
}

// State split u -> (hi, lo) and join (hi, lo) -> u over partitions with their own value offsets.
__global__ void split_join_kernel(SplitJoinArgs a) {
  for (int p = 0; p < a.npart; ++p) {
    const int64_t n = a.count[p];
    double *u = a.u + a.u_off[p];
    float *hi = a.hi + a.hi_off[p];
    float *lo = a.lo + a.lo_off[p];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      if (a.join) {
        u[i] = (double)hi[i] + (double)lo[i];
      } else {
        const double v = u[i];
        const float h = __double2float_rn(v);
        hi[i] = h;
        lo[i] = __double2float_rn(v - (double)h);
      }
    }
  }
}

}  // namespace

bool launch_rhs_mixed(int N, const MixedArgs &A, int consumer_warps, int ring_max, int num_sms, cudaStream_t st,
                      LaunchInfo *info) {
  switch (N) {
    case 1: return launch_mixed_cw<1>(A, consumer_warps, ring_max, num_sms, st, info);
    case 2: return launch_mixed_cw<2>(A, consumer_warps, ring_max, num_sms, st, info);
    case 3: return launch_mixed_cw<3>(A, consumer_warps, ring_max, num_sms, st, info);
    case 4: return launch_mixed_cw<4>(A, consumer_warps, ring_max, num_sms, st, info);
    case 5: return launch_mixed_cw<5>(A, consumer_warps, ring_max, num_sms, st, info);
    default: return false;
  }
}

void prepare_rhs_mixed(int N, int consumer_warps) {
  switch (N) {
    case 1: prepare_mixed_cw<1>(consumer_warps); break;
    case 2: prepare_mixed_cw<2>(consumer_warps); break;
    case 3: prepare_mixed_cw<3>(consumer_warps); break;
    case 4: prepare_mixed_cw<4>(consumer_warps); break;
    case 5: prepare_mixed_cw<5>(consumer_warps); break;
    default: break;
  }
}

uint32_t mixed_slot_bytes(int N) {
  switch (N) {
    case 1: return MixedCfg<1>::SLOT_B;
    case 2: return MixedCfg<2>::SLOT_B;
    case 3: return MixedCfg<3>::SLOT_B;
    case 4: return MixedCfg<4>::SLOT_B;
    case 5: return MixedCfg<5>::SLOT_B;
    default: return 0;
  }
}

template <typename T>
void launch_compact_geometry(const CompactGeoArgs<T> &g, cudaStream_t st) {
  const int threads = 128;
  const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((g.elem_total + threads - 1) / threads, 65535));
  compact_geometry_kernel<T><<<(int)blocks, threads, 0, st>>>(g);
  cuda_check(cudaGetLastError(), "compact_geometry_kernel launch");
}
template void launch_compact_geometry<float>(const CompactGeoArgs<float> &, cudaStream_t);
template void launch_compact_geometry<double>(const CompactGeoArgs<double> &, cudaStream_t);

void launch_split_join(const SplitJoinArgs &a, cudaStream_t st) {
  split_join_kernel<<<1184, 256, 0, st>>>(a);
  cuda_check(cudaGetLastError(), "split_join_kernel launch");
}

}  // namespace dgk
