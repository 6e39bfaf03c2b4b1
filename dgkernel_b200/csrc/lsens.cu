// Learned-sensor artificial viscosity on the mixed-precision stage: the shock sensor over every element, then
// the BR1 viscous term only where it is not zero.
//
// Per stage, before the tensor-core mixed stage (tcm.cu), which adds the result to its right-hand side:
//   ls_sensor   every element: modal coefficients uhat = Vinv u (FP64), the Persson-Peraire activation from
//               log10(E_top / E), the 35 -> 32 -> 32 -> 1 network (tanh, tanh, sigmoid; FP16 weights, FP32 sums)
//               on uhat / |uhat| with the PP fallback inside (lo, hi) and, in mode 3, outputs <= lo read as a
//               smooth element; eps_e = eps0 sigma_e h_e / N; elements with eps_e > 0 form the active list.
//   ls_touch    the active elements and their face neighbours are marked; ls_compact lists them (touched).
//   ls_grad     active elements: q_d = D_d u + LIFT (Fscale n_d (uP - uM) / 2) (FP64), stored as eps_e q_d.
//   ls_div      touched elements: eps_e sum_d D_d q_d + LIFT (Fscale / 2 sum_d n_d (epsP qP_d - epsM qM_d)),
//               the viscous right-hand side, with eps q = 0 on elements that are not active.
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

template <int N>
__global__ void __launch_bounds__(4 * kLsElems) ls_sensor_kernel(const LsArgs A) {
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
  for (int st = blockIdx.x; st < 2 * A.ntiles; st += gridDim.x) {
    const MTile tl = A.tiles[st >> 1];
    const int e0 = (st & 1) * kLsElems;  // half of the 128-element tile
    const int ne = max(0, min(kLsElems, tl.nelem - e0));
    const int64_t base = tl.node_base + (int64_t)e0 * NP;
    for (int x = tid; x < ne * NP; x += blockDim.x) su[x] = (double)A.uhi[base + x] + (double)A.ulo[base + x];
    __syncthreads();
    const bool valid = e < ne;
    const double *ue = su + (valid ? e : 0) * NP;
    double tot = 0.0, top = 0.0;
    double uh[(NP + 3) / 4];
#pragma unroll
    for (int k = 0; k < (NP + 3) / 4; ++k) {
      const int i = t + 4 * k;
      double s = 0.0;
      if (i < NP) {
#pragma unroll 5
        for (int j = 0; j < NP; ++j) s = fma(sVi[i * NP + j], ue[j], s);
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
      const float *x = sf + e * NPP;
#pragma unroll
      for (int k = 0; k < kLsHid / 4; ++k) {
        const int o = t + 4 * k;
        float s0 = __half2float(b1[o]), s1 = 0.f;
#pragma unroll
        for (int j = 0; j + 1 < NP; j += 2) {
          s0 = fmaf(__half2float(W1[o * NP + j]), x[j], s0);
          s1 = fmaf(__half2float(W1[o * NP + j + 1]), x[j + 1], s1);
        }
        if (NP & 1) s0 = fmaf(__half2float(W1[o * NP + NP - 1]), x[NP - 1], s0);
        sh[e * kLsHid + o] = tanhf(s0 + s1);
      }
      __syncwarp();
      float z = 0.f;
#pragma unroll
      for (int k = 0; k < kLsHid / 4; ++k) {
        const int o = t + 4 * k;
        float s0 = __half2float(b2[o]), s1 = 0.f;
#pragma unroll
        for (int j = 0; j < kLsHid; j += 2) {
          s0 = fmaf(__half2float(W2[o * kLsHid + j]), sh[e * kLsHid + j], s0);
          s1 = fmaf(__half2float(W2[o * kLsHid + j + 1]), sh[e * kLsHid + j + 1], s1);
        }
        z = fmaf(__half2float(w3[o]), tanhf(s0 + s1), z);
      }
      z += __shfl_xor_sync(0xffffffffu, z, 1);
      z += __shfl_xor_sync(0xffffffffu, z, 2);
      const float sg = 1.f / (1.f + expf(-(z + __half2float(b3[0]))));
      if (sg > A.conf_lo && sg < A.conf_hi) {
        fallback = true;  // low confidence: the PP activation stands
      } else {
        sig = (A.mode == 3 && sg <= A.conf_lo) ? 0.0 : (double)sg;
      }
    }
    if (valid && t == 0) {
      const int64_t slot = tl.elem_slot + e0 + e;
      const double eps = A.eps0 * sig * A.h_over_n[slot];
      A.eps[slot] = eps;
      int a = -1;
      if (eps > 0.0) {
        a = atomicAdd(&A.counts[0], 1);
        A.alist[a] = (int32_t)slot;
      }
      A.aslot[slot] = a;
      if (fallback) atomicAdd(&A.counts[2], 1);
    }
    __syncthreads();
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

// Sparse passes: one warp per element, lanes over the element's nodes (i = lane, lane + 32) and face points; the
// FP64 matrices are read transposed from global memory (DT[j][i], LT[m][i]: a warp's lanes read consecutive
// values, and the few tens of KB stay in L1), per-warp values in shared memory, no block barrier.
constexpr int kLsWarps = 8;  // warps (elements in flight) per block

template <int N>
__global__ void __launch_bounds__(32 * kLsWarps) ls_grad_kernel(const LsArgs A) {
  using O = Order<N>;
  constexpr int NP = O::NP, NF = O::NF;
  __shared__ double s_u[kLsWarps][NP], s_j[kLsWarps][3][NF];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double *su = s_u[w];
  const int n = *reinterpret_cast<volatile const int *>(&A.counts[0]);
  for (int a = blockIdx.x * kLsWarps + w; a < n; a += gridDim.x * kLsWarps) {
    const int64_t slot = A.alist[a];
    const int p = part_of_slot(A, slot);
    const int64_t le = slot - A.slot_prefix[p];
    const int64_t ub = A.uoff[p] + le * NP, gb = A.goff[p] + le * NP, fb = A.foff[p] + le * NF;
    for (int i = lane; i < NP; i += 32) su[i] = (double)A.uhi[ub + i] + (double)A.ulo[ub + i];
    __syncwarp();
    for (int m = lane; m < NF; m += 32) {
      const int32_t g = A.gmap[fb + m];
      const double uM = su[A.fmask[m]];
      double uP = uM;
      if ((uint64_t)(int64_t)g < (uint64_t)A.n_u_values) {
        uP = (double)A.uhi[g] + (double)A.ulo[g];
      } else {
        atomicExch(A.status, kStatusBadGather);
      }
      const double jump = 0.5 * (uP - uM) * A.face[3][fb + m];
      for (int d = 0; d < 3; ++d) s_j[w][d][m] = A.face[d][fb + m] * jump;
    }
    __syncwarp();
    const double eps = A.eps[slot];
    for (int i = lane; i < NP; i += 32) {
      double ur = 0.0, us = 0.0, ut = 0.0;
#pragma unroll 5
      for (int j = 0; j < NP; ++j) {
        const double v = su[j];
        ur = fma(__ldg(A.Dr + j * NP + i), v, ur);
        us = fma(__ldg(A.Ds + j * NP + i), v, us);
        ut = fma(__ldg(A.Dt + j * NP + i), v, ut);
      }
      double q[3];
      for (int d = 0; d < 3; ++d) q[d] = A.geo[d][gb + i] * ur + A.geo[3 + d][gb + i] * us + A.geo[6 + d][gb + i] * ut;
#pragma unroll 6
      for (int m = 0; m < NF; ++m) {
        const double l = __ldg(A.LIFT + m * NP + i);
        q[0] = fma(l, s_j[w][0][m], q[0]);
        q[1] = fma(l, s_j[w][1][m], q[1]);
        q[2] = fma(l, s_j[w][2][m], q[2]);
      }
      for (int d = 0; d < 3; ++d) A.eq[((int64_t)a * 3 + d) * NP + i] = eps * q[d];
    }
    __syncwarp();
  }
}

template <int N>
__global__ void __launch_bounds__(32 * kLsWarps) ls_div_kernel(const LsArgs A) {
  using O = Order<N>;
  constexpr int NP = O::NP, NF = O::NF;
  __shared__ double s_q[kLsWarps][3][NP], s_f[kLsWarps][NF];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int n = *reinterpret_cast<volatile const int *>(&A.counts[1]);
  for (int r = blockIdx.x * kLsWarps + w; r < n; r += gridDim.x * kLsWarps) {
    const int64_t slot = A.tlist[r];
    const int p = part_of_slot(A, slot);
    const int64_t le = slot - A.slot_prefix[p];
    const int64_t gb = A.goff[p] + le * NP, fb = A.foff[p] + le * NF;
    const int a = A.aslot[slot];
    for (int i = lane; i < NP; i += 32)
      for (int d = 0; d < 3; ++d) s_q[w][d][i] = a >= 0 ? A.eq[((int64_t)a * 3 + d) * NP + i] : 0.0;
    __syncwarp();
    for (int m = lane; m < NF; m += 32) {
      const int32_t g = A.gmap[fb + m];
      const int jM = A.fmask[m];
      double ePq[3] = {0.0, 0.0, 0.0};
      int node;
      const int64_t ns = ((uint64_t)(int64_t)g < (uint64_t)A.n_u_values) ? slot_of_value(A, g, NP, &node) : -1;
      if (ns >= 0) {
        const int an = A.aslot[ns];
        if (an >= 0)
          for (int d = 0; d < 3; ++d) ePq[d] = A.eq[((int64_t)an * 3 + d) * NP + node];
      } else {
        atomicExch(A.status, kStatusBadGather);
      }
      double v = 0.0;
      for (int d = 0; d < 3; ++d) v += A.face[d][fb + m] * (ePq[d] - s_q[w][d][jM]);
      s_f[w][m] = 0.5 * A.face[3][fb + m] * v;
    }
    __syncwarp();
    for (int i = lane; i < NP; i += 32) {
      double div = 0.0;
      if (a >= 0) {
        double qr[3] = {0.0, 0.0, 0.0}, qs[3] = {0.0, 0.0, 0.0}, qt[3] = {0.0, 0.0, 0.0};
#pragma unroll 5
        for (int j = 0; j < NP; ++j) {
          const double dr = __ldg(A.Dr + j * NP + i), ds = __ldg(A.Ds + j * NP + i), dt = __ldg(A.Dt + j * NP + i);
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            const double v = s_q[w][d][j];
            qr[d] = fma(dr, v, qr[d]);
            qs[d] = fma(ds, v, qs[d]);
            qt[d] = fma(dt, v, qt[d]);
          }
        }
        for (int d = 0; d < 3; ++d)
          div += A.geo[d][gb + i] * qr[d] + A.geo[3 + d][gb + i] * qs[d] + A.geo[6 + d][gb + i] * qt[d];
      }
      double lift = 0.0;
#pragma unroll 6
      for (int m = 0; m < NF; ++m) lift = fma(__ldg(A.LIFT + m * NP + i), s_f[w][m], lift);
      A.visc[(int64_t)r * NP + i] = div + lift;
    }
    __syncwarp();
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
  ls_grad_kernel<N><<<num_sms * 8, 32 * kLsWarps, 0, st>>>(A);
  cuda_check(cudaGetLastError(), "ls_grad_kernel launch");
  ls_div_kernel<N><<<num_sms * 8, 32 * kLsWarps, 0, st>>>(A);
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
