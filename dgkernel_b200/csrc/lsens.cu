// Learned-sensor artificial viscosity on the mixed-precision stage: the shock sensor over every element, then
// the BR1 viscous term only where it is not zero.
//
// Per stage, before the tensor-core mixed stage (tcm.cu), which adds the result to its right-hand side:
//   ls_sensor   every element: modal coefficients uhat = Vinv u (FP64, on the FP64 tensor path), the
//               Persson-Peraire activation from log10(E_top / E), the 35 -> 32 -> 32 -> 1 network (tanh, tanh,
//               sigmoid; FP16 weights, FP32 sums; its hidden layers as TF32 tensor products with two-part
//               inputs) on uhat / |uhat| with the PP fallback inside (lo, hi) and, in mode 3, outputs <= lo read
//               as a smooth element; eps_e = eps0 sigma_e h_e / N; elements with eps_e > 0 form the active list.
//   ls_touch    the active elements and their face neighbours are marked; ls_compact lists them (touched).
//   ls_grad     active elements: q_d = D_d u + LIFT (Fscale n_d (uP - uM) / 2) (FP64 tensor path), stored as
//               eps_e q_d.
//   ls_div      touched elements: sum_d d/dx_d (eps_e q_d) + LIFT (Fscale / 2 sum_d n_d (epsP qP_d - epsM qM_d)),
//               the viscous right-hand side, with eps q = 0 on elements that are not active; on straight-sided
//               elements the derivative is sum_k D_k (sum_d (d xi_k / d x_d) eps q_d) (FP64 tensor path).
// This is the BR1 viscosity of the plain viscosity stage (av.cu) restricted to where it is not zero: an element
// whose own and neighbours' eps vanish gets no viscous term there either.  The sparse passes walk device-side
// counts with persistent grids, so a stage needs no host synchronisation.
#include <cuda_fp16.h>

#include <algorithm>
#include <cstdint>

#include "dg_kernels.cuh"
#include "kernels.hpp"
#include "runner.hpp"

namespace dgk {

namespace {

constexpr int kLsHid = 32;
constexpr int kLsElems = 64;   // sensor pass: elements per block, 4 threads each

__host__ __device__ constexpr int ls_mlp_params(int nin) {
  return kLsHid * nin + kLsHid + kLsHid * kLsHid + kLsHid + kLsHid + 1;
}

__device__ __forceinline__ double ls_pp_sigma(double S, double s0, double kappa) {
  if (!(S >= s0 - kappa)) return 0.0;
  if (S > s0 + kappa) return 1.0;
  return 0.5 * (1.0 + sin(3.141592653589793 * (S - s0) / (2.0 * kappa)));
}

// partition of an element slot (slot_prefix ascending)
__device__ __forceinline__ int part_of_slot(const LsArgs &A, int64_t slot) {
  int p = 0;
  while (p + 1 < A.npart && A.slot_prefix[p + 1] <= slot) ++p;
  return p;
}

// element slot and local node of a state value index; -1 when it lies in no partition
__device__ __forceinline__ int64_t slot_of_value(const LsArgs &A, int64_t g, int np, int *node) {
  for (int p = 0; p < A.npart; ++p) {
    const int64_t rel = g - A.uoff[p];
    if (rel >= 0 && rel < A.kpart[p] * np) {
      const int64_t le = rel / np;
      *node = (int)(rel - le * np);
      return A.slot_prefix[p] + le;
    }
  }
  *node = 0;
  return -1;
}

// TF32 helpers of the network's tensor products: x = hi + lo with both parts TF32 (round to nearest), an FP16
// weight as its exact TF32 bit pattern (0 outside the matrix), and one m16n8k8 product accumulated into d.
__device__ __forceinline__ void ls_tf32_split(float x, uint32_t &hi, uint32_t &lo) {
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(x));
  const float r = x - __uint_as_float(hi);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(r));
}

__device__ __forceinline__ uint32_t ls_tf32_w(const __half *W, int i, bool in) {
  return in ? __float_as_uint(__half2float(W[i])) : 0u;
}

__device__ __forceinline__ void ls_mma_tf32(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
               "{%0,%1,%2,%3};"
               : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

template <int N>
__global__ void __launch_bounds__(4 * kLsElems, 3) ls_sensor_kernel(const LsArgs A) {
  using O = Order<N>;
  constexpr int NP = O::NP;
  constexpr int NPP = NP + 1;  // padded row of the feature buffer
  extern __shared__ __align__(16) unsigned char sm[];
  double *sVi = reinterpret_cast<double *>(sm);     // [NP][NP]
  double *su = sVi + NP * NP;                       // [64][NP]
  float *sf = reinterpret_cast<float *>(su + kLsElems * NP);  // [64][NPP] features
  float *sh = sf + kLsElems * NPP;                  // [64][32] first hidden layer
  __half *sW = reinterpret_cast<__half *>(sh + kLsElems * kLsHid);
  int *sTop = reinterpret_cast<int *>(sW + ((ls_mlp_params(NP) + 7) & ~7));
  const int tid = threadIdx.x, e = tid >> 2, t = tid & 3;
  for (int x = tid; x < NP * NP; x += blockDim.x) sVi[x] = A.Vinv[x];
  for (int x = tid; x < NP; x += blockDim.x) sTop[x] = A.top[x];
  if (A.mode >= 2)
    for (int x = tid; x < ls_mlp_params(NP); x += blockDim.x) sW[x] = __ushort_as_half(A.mlp16[x]);
  __syncthreads();
  const __half *W1 = sW, *b1 = W1 + kLsHid * NP, *W2 = b1 + kLsHid, *b2 = W2 + kLsHid * kLsHid, *w3 = b2 + kLsHid,
               *b3 = w3 + kLsHid;
  // Every warp walks its own groups of 8 elements (16 per 128-element tile) in rows 8 w .. 8 w + 7 of the
  // block's buffers, with no block barrier; the state of its next group, the group's first element slot and
  // (lanes 0..7) its elements' h / N are loaded into registers while the current one is computed.
  const int lane = tid & 31, w0 = (tid >> 5) * 8, nw = blockDim.x >> 5;
  const int ngroups = 16 * A.ntiles;
  constexpr int FILL = (8 * NP + 31) / 32;  // values per lane
  float fh[FILL], fl[FILL];
  int64_t nslot = 0;
  int nne = 0;
  double nh = 0.0;
  auto load = [&](int gi) {
    const MTile tl = A.tiles[gi >> 4];
    const int e0 = (gi & 15) * 8;
    const int ne = max(0, min(8, tl.nelem - e0));
    const int64_t base = tl.node_base + (int64_t)e0 * NP;
#pragma unroll
    for (int q = 0; q < FILL; ++q) {
      const int x = lane + 32 * q;
      fh[q] = x < ne * NP ? A.uhi[base + x] : 0.f;
      fl[q] = x < ne * NP ? A.ulo[base + x] : 0.f;
    }
    nslot = tl.elem_slot + e0;
    nne = ne;
    nh = lane < ne ? A.h_over_n[nslot + lane] : 0.0;
  };
  const int g0 = blockIdx.x * nw + (tid >> 5), gstep = gridDim.x * nw;
  if (g0 < ngroups) load(g0);
  for (int gi = g0; gi < ngroups; gi += gstep) {
    const int64_t slot0 = nslot;  // this group's first element slot, its element count and h / N (lanes 0..7)
    const int ne = nne;
    const double hg = nh;
#pragma unroll
    for (int q = 0; q < FILL; ++q) {
      const int x = lane + 32 * q;
      if (x < 8 * NP) su[w0 * NP + x] = (double)fh[q] + (double)fl[q];
    }
    __syncwarp();
    if (gi + gstep < ngroups) load(gi + gstep);
    if (ne == 0) continue;  // past the tile's last element (warp-uniform)
    const bool valid = (e & 7) < ne;
    // modal coefficients uhat = Vinv u of this warp's 8 elements on the FP64 tensor path (mma.sync m8n8k4):
    // A = Vinv (8-row m-tiles, 4-column k-steps), B = the elements' nodal values (one element per column);
    // they overwrite the warp's own rows of su
    {
      constexpr int MT = (NP + 7) / 8, KT = (NP + 3) / 4;
      const int ar = lane >> 2, ac = lane & 3, be = w0 + (lane >> 2);
      double c[MT][2];
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) c[mt][0] = c[mt][1] = 0.0;
#pragma unroll
      for (int kk = 0; kk < KT; ++kk) {
        const int j = 4 * kk + ac;
        const double bv = (j < NP && ar < ne) ? su[be * NP + j] : 0.0;
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
          const int r = 8 * mt + ar;
          const double av = (r < NP && j < NP) ? sVi[r * NP + j] : 0.0;
          asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                       : "+d"(c[mt][0]), "+d"(c[mt][1])
                       : "d"(av), "d"(bv));
        }
      }
      __syncwarp();  // every lane's reads of the nodal values are done
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        const int r = 8 * mt + ar;
#pragma unroll
        for (int h = 0; h < 2; ++h)
          if (r < NP) su[(w0 + 2 * ac + h) * NP + r] = c[mt][h];
      }
      __syncwarp();
    }
    const double *ue = su + (valid ? e : w0) * NP;  // now the element's modal coefficients
    double tot = 0.0, top = 0.0;
    double uh[(NP + 3) / 4];
#pragma unroll
    for (int k = 0; k < (NP + 3) / 4; ++k) {
      const int i = t + 4 * k;
      double s = 0.0;
      if (i < NP) {
        s = ue[i];
        tot = fma(s, s, tot);
        if (sTop[i]) top = fma(s, s, top);
      }
      uh[k] = s;
    }
    tot += __shfl_xor_sync(0xffffffffu, tot, 1);
    tot += __shfl_xor_sync(0xffffffffu, tot, 2);
    top += __shfl_xor_sync(0xffffffffu, top, 1);
    top += __shfl_xor_sync(0xffffffffu, top, 2);
    const double S = tot > 0.0 ? log10(top / tot) : -INFINITY;
    double sig = A.mode == 0 ? 0.0 : ls_pp_sigma(S, A.s0, A.kappa);
    bool fallback = false;
    if (A.mode >= 2) {
      const double inv = tot > 0.0 ? 1.0 / sqrt(tot) : 0.0;
#pragma unroll
      for (int k = 0; k < (NP + 3) / 4; ++k) {
        const int i = t + 4 * k;
        if (i < NP) sf[e * NPP + i] = (float)(uh[k] * inv);
      }
      __syncwarp();
      // the network on the warp's 8 elements with tensor products (mma.sync m16n8k8, TF32 operands, FP32
      // sums): every FP16 weight is exact in TF32 and each FP32 input is split into two TF32 parts (hi + lo),
      // so the products keep FP32-level rounding.  Rows are hidden units (two 16-row m-tiles), columns the
      // warp's elements; lane (g = l / 4, c = l mod 4) holds units g, g + 8 (+16) of elements 2c, 2c + 1.
      const int g = lane >> 2, c = lane & 3;
      float o2[2][4];  // second-layer pre-activations: [m-tile][fragment]
      {
        float o1[2][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
          const float blo = __half2float(b1[16 * mt + g]), bhi = __half2float(b1[16 * mt + g + 8]);
          o1[mt][0] = o1[mt][1] = blo;
          o1[mt][2] = o1[mt][3] = bhi;
        }
#pragma unroll
        for (int kk = 0; kk < (NP + 7) / 8; ++kk) {
          const int j0 = 8 * kk + c, j1 = j0 + 4;
          const float x0 = j0 < NP ? sf[(w0 + g) * NPP + j0] : 0.f, x1 = j1 < NP ? sf[(w0 + g) * NPP + j1] : 0.f;
          uint32_t bh[2], bl[2];
          ls_tf32_split(x0, bh[0], bl[0]);
          ls_tf32_split(x1, bh[1], bl[1]);
#pragma unroll
          for (int mt = 0; mt < 2; ++mt) {
            const int r0 = 16 * mt + g;
            const uint32_t a[4] = {ls_tf32_w(W1, r0 * NP + j0, j0 < NP), ls_tf32_w(W1, (r0 + 8) * NP + j0, j0 < NP),
                                   ls_tf32_w(W1, r0 * NP + j1, j1 < NP), ls_tf32_w(W1, (r0 + 8) * NP + j1, j1 < NP)};
            ls_mma_tf32(o1[mt], a, bh);
            ls_mma_tf32(o1[mt], a, bl);
          }
        }
        // first hidden layer -> shared memory [element][unit], the second layer's inputs
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
          for (int f = 0; f < 4; ++f)
            sh[(w0 + 2 * c + (f & 1)) * kLsHid + 16 * mt + g + 8 * (f >> 1)] = tanhf(o1[mt][f]);
        __syncwarp();
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
          const float blo = __half2float(b2[16 * mt + g]), bhi = __half2float(b2[16 * mt + g + 8]);
          o2[mt][0] = o2[mt][1] = blo;
          o2[mt][2] = o2[mt][3] = bhi;
        }
#pragma unroll
        for (int kk = 0; kk < kLsHid / 8; ++kk) {
          const int j0 = 8 * kk + c, j1 = j0 + 4;
          uint32_t bh[2], bl[2];
          ls_tf32_split(sh[(w0 + g) * kLsHid + j0], bh[0], bl[0]);
          ls_tf32_split(sh[(w0 + g) * kLsHid + j1], bh[1], bl[1]);
#pragma unroll
          for (int mt = 0; mt < 2; ++mt) {
            const int r0 = 16 * mt + g;
            const uint32_t a[4] = {ls_tf32_w(W2, r0 * kLsHid + j0, true), ls_tf32_w(W2, (r0 + 8) * kLsHid + j0, true),
                                   ls_tf32_w(W2, r0 * kLsHid + j1, true), ls_tf32_w(W2, (r0 + 8) * kLsHid + j1, true)};
            ls_mma_tf32(o2[mt], a, bh);
            ls_mma_tf32(o2[mt], a, bl);
          }
        }
      }
      // output unit: this lane's four units for elements 2c and 2c + 1, summed over the lanes of the same c
      float za = 0.f, zb = 0.f;
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const float wlo = __half2float(w3[16 * mt + g]), whi = __half2float(w3[16 * mt + g + 8]);
        za += wlo * tanhf(o2[mt][0]) + whi * tanhf(o2[mt][2]);
        zb += wlo * tanhf(o2[mt][1]) + whi * tanhf(o2[mt][3]);
      }
#pragma unroll
      for (int m = 4; m <= 16; m <<= 1) {
        za += __shfl_xor_sync(0xffffffffu, za, m);
        zb += __shfl_xor_sync(0xffffffffu, zb, m);
      }
      const int el = e & 7;  // this thread's element: held by lane el / 2 (c = el / 2, g = 0)
      const float zsa = __shfl_sync(0xffffffffu, za, el >> 1), zsb = __shfl_sync(0xffffffffu, zb, el >> 1);
      const float z = (el & 1) ? zsb : zsa;
      const float sg = 1.f / (1.f + expf(-(z + __half2float(b3[0]))));
      if (sg > A.conf_lo && sg < A.conf_hi) {
        fallback = true;  // low confidence: the PP activation stands
      } else {
        sig = (A.mode == 3 && sg <= A.conf_lo) ? 0.0 : (double)sg;
      }
    }
    const double hh = __shfl_sync(0xffffffffu, hg, e & 7);  // this element's h / N
    if (valid && t == 0) {
      const int64_t slot = slot0 + (e & 7);
      const double eps = A.eps0 * sig * hh;
      A.eps[slot] = eps;
      int a = -1;
      if (eps > 0.0) {
        a = atomicAdd(&A.counts[0], 1);
        A.alist[a] = (int32_t)slot;
      }
      A.aslot[slot] = a;
      if (fallback) atomicAdd(&A.counts[2], 1);
    }
    __syncwarp();  // the warp's rows are free for its next group
  }
}

// the active elements and their face neighbours
__global__ void ls_touch_kernel(const LsArgs A, int np) {
  const int n = *reinterpret_cast<volatile const int *>(&A.counts[0]);
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    const int64_t slot = A.alist[a];
    A.tflag[slot] = 1;
    for (int f = 0; f < 4; ++f) {
      int node;
      const int64_t ns = slot_of_value(A, (int64_t)(uint32_t)A.conn[slot * kMixedConnWords + f], np, &node);
      if (ns >= 0) A.tflag[ns] = 1;
    }
  }
}

// touched list and row of every slot (-1 elsewhere); the flags are cleared for the next stage
__global__ void ls_compact_kernel(const LsArgs A) {
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < A.nslots; s += (int64_t)gridDim.x * blockDim.x) {
    if (A.tflag[s]) {
      const int r = atomicAdd(&A.counts[1], 1);
      A.tlist[r] = (int32_t)s;
      A.vslot[s] = r;
      A.tflag[s] = 0;
    } else {
      A.vslot[s] = -1;
    }
  }
}

// Sparse passes: one block of MT warps per group of 8 listed elements (the n-tile of the FP64 tensor path,
// mma.sync m8n8k4).  The block stages the group in shared memory (per-element offsets, eps and metrics; nodal
// values; face terms: each thread's few face points with their loads issued together), then warp mt applies the
// element matrices to rows 8 mt .. 8 mt + 7, reading their fragments transposed through L1 (DT[j][i], LT[m][i]:
// the few tens of KB stay there); lane l's output row is 8 mt + l / 4, its elements 2 (l mod 4) and
// 2 (l mod 4) + 1.  The mixed stage requires straight-sided elements, so the metrics are constant over an
// element and are read once per element.
__device__ __forceinline__ void ls_dmma(double &c0, double &c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

template <int N>
struct LsCfg {
  using O = Order<N>;
  static constexpr int NP = O::NP, NF = O::NF;
  static constexpr int MT = (NP + 7) / 8, KT = (NP + 3) / 4, KL = NF / 4;
  static constexpr int NPU = 4 * KT;  // padded node rows of a staged element
  static constexpr int THREADS = 32 * MT;
  static constexpr int QF = (8 * NF + THREADS - 1) / THREADS;  // face points per thread
  static_assert(NF % 4 == 0, "face points in whole k-steps");
};

// per-element data of a staged group
struct LsElem {
  int64_t ub, fb;   // value offsets of the element in the state and face arrays
  double geo[9];    // rx .. tz (constant over a straight-sided element)
  double eps;
  int ok, act;      // listed element; row in the active list (-1: not active)
};

template <int N>
__device__ __forceinline__ void ls_stage_elems(const LsArgs &A, const int32_t *list, int n, int gi, LsElem *se,
                                               bool with_geo) {
  using C = LsCfg<N>;
  constexpr int NP = C::NP, NF = C::NF;
  const int t = threadIdx.x;
  if (t < 8) {
    LsElem x{};
    x.act = -1;
    if (8 * gi + t < n) {
      const int64_t slot = list[8 * gi + t];
      const int p = part_of_slot(A, slot);
      const int64_t le = slot - A.slot_prefix[p];
      x.ub = A.uoff[p] + le * NP;
      x.fb = A.foff[p] + le * NF;
      const int64_t gb = A.goff[p] + le * NP;
      if (with_geo)
        for (int m = 0; m < 9; ++m) x.geo[m] = A.geo[m][gb];
      x.eps = A.eps[slot];
      x.act = A.aslot[slot];
      x.ok = 1;
    }
    se[t] = x;
  }
}

template <int N>
__global__ void __launch_bounds__(LsCfg<N>::THREADS) ls_grad_kernel(const LsArgs A) {
  using C = LsCfg<N>;
  constexpr int NP = C::NP, NF = C::NF, KT = C::KT, KL = C::KL, NPU = C::NPU, QF = C::QF;
  __shared__ double su[8 * NPU], sj[3 * 8 * NF];
  __shared__ LsElem se[8];
  const int tid = threadIdx.x, lane = tid & 31, mt = tid >> 5;
  const int ar = lane >> 2, ac = lane & 3, r = 8 * mt + ar;
  const int n = *reinterpret_cast<volatile const int *>(&A.counts[0]);
  const int ngroups = (n + 7) / 8;
  for (int gi = blockIdx.x; gi < ngroups; gi += gridDim.x) {
    ls_stage_elems<N>(A, A.alist, n, gi, se, true);
    __syncthreads();
    for (int x = tid; x < 8 * NPU; x += C::THREADS) {
      const int e = x / NPU, i = x - e * NPU;
      su[x] = (se[e].ok && i < NP) ? (double)A.uhi[se[e].ub + i] + (double)A.ulo[se[e].ub + i] : 0.0;
    }
    // this thread's face points: gather indices and face data, then the neighbour traces
    int32_t g[QF];
    double nd[QF][4];
    bool use[QF];
#pragma unroll
    for (int b = 0; b < QF; ++b) {
      const int x = tid + C::THREADS * b, e = min(x / NF, 7), m = x - e * NF;
      use[b] = x < 8 * NF && se[e].ok;
      g[b] = use[b] ? A.gmap[se[e].fb + m] : 0;
      // straight-sided elements: normals and Fscale are constant over a face (its first point's values)
      for (int d = 0; d < 4; ++d) nd[b][d] = use[b] ? A.face[d][se[e].fb + (m / (NF / 4)) * (NF / 4)] : 0.0;
    }
    float ph[QF], pl[QF];
#pragma unroll
    for (int b = 0; b < QF; ++b) {
      const bool in = use[b] && (uint64_t)(int64_t)g[b] < (uint64_t)A.n_u_values;
      if (use[b] && !in) {
        atomicExch(A.status, kStatusBadGather);
        g[b] = -1;  // rejected index: the interior trace stands
      }
      ph[b] = in ? A.uhi[g[b]] : 0.f;
      pl[b] = in ? A.ulo[g[b]] : 0.f;
    }
    __syncthreads();  // su complete
#pragma unroll
    for (int b = 0; b < QF; ++b) {
      const int x = tid + C::THREADS * b;
      if (x < 8 * NF) {
        const int e = x / NF, m = x - e * NF;
        double jump = 0.0;
        if (use[b]) {
          const double uM = su[e * NPU + A.fmask[m]];
          const double uP = g[b] < 0 ? uM : (double)ph[b] + (double)pl[b];
          jump = 0.5 * (uP - uM) * nd[b][3];
        }
        for (int d = 0; d < 3; ++d) sj[(d * 8 + e) * NF + m] = nd[b][d] * jump;
      }
    }
    __syncthreads();  // sj complete
    double cr[2] = {0.0, 0.0}, cs[2] = {0.0, 0.0}, ct[2] = {0.0, 0.0};
    double cl[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
    for (int kk = 0; kk < KT; ++kk) {
      const int j = 4 * kk + ac;
      const bool in = r < NP && j < NP;
      const double bv = su[ar * NPU + j];
      ls_dmma(cr[0], cr[1], in ? __ldg(A.Dr + j * NP + r) : 0.0, bv);
      ls_dmma(cs[0], cs[1], in ? __ldg(A.Ds + j * NP + r) : 0.0, bv);
      ls_dmma(ct[0], ct[1], in ? __ldg(A.Dt + j * NP + r) : 0.0, bv);
    }
#pragma unroll 5
    for (int kk = 0; kk < KL; ++kk) {
      const int m = 4 * kk + ac;
      const double al = r < NP ? __ldg(A.LIFT + m * NP + r) : 0.0;
#pragma unroll
      for (int d = 0; d < 3; ++d) ls_dmma(cl[d][0], cl[d][1], al, sj[(d * 8 + ar) * NF + m]);
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int e = 2 * ac + h;
      if (r < NP && se[e].ok) {
        const LsElem &x = se[e];
        for (int d = 0; d < 3; ++d) {
          const double q = x.geo[d] * cr[h] + x.geo[3 + d] * cs[h] + x.geo[6 + d] * ct[h] + cl[d][h];
          A.eq[((int64_t)(8 * gi + e) * NP + r) * 3 + d] = x.eps * q;
        }
      }
    }
    __syncthreads();  // the staging buffers are free for the next group
  }
}

template <int N>
__global__ void __launch_bounds__(LsCfg<N>::THREADS) ls_div_kernel(const LsArgs A) {
  using C = LsCfg<N>;
  constexpr int NP = C::NP, NF = C::NF, KT = C::KT, KL = C::KL, NPU = C::NPU, QF = C::QF;
  __shared__ double sq[3 * 8 * NPU], sf[8 * NF];
  __shared__ LsElem se[8];
  const int tid = threadIdx.x, lane = tid & 31, mt = tid >> 5;
  const int ar = lane >> 2, ac = lane & 3, r = 8 * mt + ar;
  const int n = *reinterpret_cast<volatile const int *>(&A.counts[1]);
  const int ngroups = (n + 7) / 8;
  for (int gi = blockIdx.x; gi < ngroups; gi += gridDim.x) {
    ls_stage_elems<N>(A, A.tlist, n, gi, se, true);
    __syncthreads();
    // the group's eps q_d, and this thread's face points: gather indices and face data
    for (int x = tid; x < 3 * 8 * NPU; x += C::THREADS) {  // node-major reads: a node's 3 values are adjacent
      const int e = x / (3 * NPU), y = x - e * 3 * NPU, i = y / 3, d = y - 3 * i;
      const int ae = se[e].act;
      sq[(d * 8 + e) * NPU + i] = (ae >= 0 && i < NP) ? A.eq[((int64_t)ae * NP + i) * 3 + d] : 0.0;
    }
    int32_t g[QF];
    double nd[QF][4];
    bool use[QF];
#pragma unroll
    for (int b = 0; b < QF; ++b) {
      const int x = tid + C::THREADS * b, e = min(x / NF, 7), m = x - e * NF;
      use[b] = x < 8 * NF && se[e].ok;
      g[b] = use[b] ? A.gmap[se[e].fb + m] : 0;
      // straight-sided elements: normals and Fscale are constant over a face (its first point's values)
      for (int d = 0; d < 4; ++d) nd[b][d] = use[b] ? A.face[d][se[e].fb + (m / (NF / 4)) * (NF / 4)] : 0.0;
    }
    // the neighbours' rows in the active list, then their eps q
    int an[QF], node[QF];
#pragma unroll
    for (int b = 0; b < QF; ++b) {
      an[b] = -1;
      node[b] = 0;
      if (use[b]) {
        const int64_t ns =
            ((uint64_t)(int64_t)g[b] < (uint64_t)A.n_u_values) ? slot_of_value(A, g[b], NP, &node[b]) : -1;
        if (ns >= 0)
          an[b] = A.aslot[ns];
        else
          atomicExch(A.status, kStatusBadGather);
      }
    }
    double ePq[QF][3];
#pragma unroll
    for (int b = 0; b < QF; ++b)
#pragma unroll
      for (int d = 0; d < 3; ++d) ePq[b][d] = an[b] >= 0 ? A.eq[((int64_t)an[b] * NP + node[b]) * 3 + d] : 0.0;
    __syncthreads();  // sq complete
#pragma unroll
    for (int b = 0; b < QF; ++b) {
      const int x = tid + C::THREADS * b;
      if (x < 8 * NF) {
        const int e = x / NF, m = x - e * NF;
        double flux = 0.0;
        if (use[b]) {
          const int jM = A.fmask[m];
          double v = 0.0;
          for (int d = 0; d < 3; ++d) v += nd[b][d] * (ePq[b][d] - sq[(d * 8 + e) * NPU + jM]);
          flux = 0.5 * nd[b][3] * v;
        }
        sf[e * NF + m] = flux;
      }
    }
    __syncthreads();  // every surface flux formed from sq
    // div(eps q) = sum_k D_k a_k with a_k = sum_d (d xi_k / d x_d) eps q_d (metrics constant over the element);
    // a_k replaces eps q_d in place, each thread owning whole nodes
    bool any_active = false;
    for (int e = 0; e < 8; ++e) any_active |= se[e].act >= 0;
    if (any_active) {
      for (int y = tid; y < 8 * NPU; y += C::THREADS) {
        const int e = y / NPU;
        if (se[e].act >= 0) {
          const double q0 = sq[y], q1 = sq[8 * NPU + y], q2 = sq[16 * NPU + y];
#pragma unroll
          for (int k = 0; k < 3; ++k)
            sq[k * 8 * NPU + y] = se[e].geo[3 * k] * q0 + se[e].geo[3 * k + 1] * q1 + se[e].geo[3 * k + 2] * q2;
        }
      }
      __syncthreads();
    }
    double c[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}}, cl[2] = {0.0, 0.0};
    if (any_active) {
#pragma unroll
      for (int kk = 0; kk < KT; ++kk) {
        const int j = 4 * kk + ac;
        const bool in = r < NP && j < NP;
        ls_dmma(c[0][0], c[0][1], in ? __ldg(A.Dr + j * NP + r) : 0.0, sq[ar * NPU + j]);
        ls_dmma(c[1][0], c[1][1], in ? __ldg(A.Ds + j * NP + r) : 0.0, sq[(8 + ar) * NPU + j]);
        ls_dmma(c[2][0], c[2][1], in ? __ldg(A.Dt + j * NP + r) : 0.0, sq[(16 + ar) * NPU + j]);
      }
    }
#pragma unroll 5
    for (int kk = 0; kk < KL; ++kk) {
      const int m = 4 * kk + ac;
      ls_dmma(cl[0], cl[1], r < NP ? __ldg(A.LIFT + m * NP + r) : 0.0, sf[ar * NF + m]);
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int e = 2 * ac + h;
      if (r < NP && se[e].ok) A.visc[(int64_t)(8 * gi + e) * NP + r] = (c[0][h] + c[1][h] + c[2][h]) + cl[h];
    }
    __syncthreads();  // the staging buffers are free for the next group
  }
}

template <int N>
size_t ls_sensor_smem() {
  constexpr int NP = Order<N>::NP;
  return sizeof(double) * (NP * NP + kLsElems * NP) + sizeof(float) * (kLsElems * (NP + 1) + kLsElems * kLsHid) +
         sizeof(__half) * ((ls_mlp_params(NP) + 7) & ~7) + sizeof(int) * NP;
}

template <int N>
void ls_attrs() {
  static bool done[64] = {};
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev >= 0 && dev < 64 && done[dev]) return;
  cuda_check(cudaFuncSetAttribute(ls_sensor_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)ls_sensor_smem<N>()),
             "ls_sensor smem");
  if (dev >= 0 && dev < 64) done[dev] = true;
}

template <int N>
void launch_ls_n(const LsArgs &A, int num_sms, cudaStream_t st) {
  ls_attrs<N>();
  cuda_check(cudaMemsetAsync(A.counts, 0, 3 * sizeof(int32_t), st), "reset counts");
  const int gs = std::max(1, std::min(2 * A.ntiles, num_sms * 8));
  ls_sensor_kernel<N><<<gs, 4 * kLsElems, ls_sensor_smem<N>(), st>>>(A);
  cuda_check(cudaGetLastError(), "ls_sensor_kernel launch");
  ls_touch_kernel<<<num_sms * 2, 256, 0, st>>>(A, Order<N>::NP);
  cuda_check(cudaGetLastError(), "ls_touch_kernel launch");
  ls_compact_kernel<<<num_sms * 4, 256, 0, st>>>(A);
  cuda_check(cudaGetLastError(), "ls_compact_kernel launch");
  ls_grad_kernel<N><<<num_sms * 8, LsCfg<N>::THREADS, 0, st>>>(A);
  cuda_check(cudaGetLastError(), "ls_grad_kernel launch");
  ls_div_kernel<N><<<num_sms * 8, LsCfg<N>::THREADS, 0, st>>>(A);
  cuda_check(cudaGetLastError(), "ls_div_kernel launch");
}

}  // namespace

bool ls_supported(int N) { return N >= 1 && N <= 4; }

void prepare_ls(int N) {
  switch (N) {
    case 1: ls_attrs<1>(); break;
    case 2: ls_attrs<2>(); break;
    case 3: ls_attrs<3>(); break;
    case 4: ls_attrs<4>(); break;
    default: break;
  }
}

void launch_ls(int N, const LsArgs &A, int num_sms, cudaStream_t st) {
  switch (N) {
    case 1: launch_ls_n<1>(A, num_sms, st); break;
    case 2: launch_ls_n<2>(A, num_sms, st); break;
    case 3: launch_ls_n<3>(A, num_sms, st); break;
    case 4: launch_ls_n<4>(A, num_sms, st); break;
    default: throw Error(DGK_ERR_UNSUPPORTED, "learned-sensor viscosity: orders 1..4");
  }
}

}  // namespace dgk
