// Artificial-viscosity stage with a modal shock sensor, and the sensor's small MLP (training and inference).
//
// Sensor (Persson & Peraire): per element the modal coefficients uhat = Vinv u (orthonormal simplex modes,
// order i, j, k), S = log10(energy of the modes of total degree N / total energy), activation
// sigma = 0 below s0 - kappa, 1 above s0 + kappa, (1 + sin(pi (S - s0) / (2 kappa))) / 2 between.  Learned
// sensor: sigma = MLP(uhat / |uhat|), a 35 -> 32 -> 32 -> 1 network (tanh, tanh, sigmoid) with FP16 weights and
// FP32 sums; where its output lies inside the low-confidence band (lo, hi) the element falls back to the PP
// activation.  Viscosity eps_e = eps0 sigma_e h_e / N, h_e = 2 / max Fscale over the element's face points.
//
// Viscous term (BR1 with central fluxes): q_d = D_d u + LIFT (Fscale n_d (uP - uM) / 2), d = x, y, z, then
// rhs += eps_e sum_d D_d q_d + LIFT (Fscale 1/2 sum_d n_d (epsP qP_d - epsM qM_d)), added to the
// Lax-Friedrichs right-hand side of the plain stage; the LSERK4 update follows in the same kernel.
//
// Two kernels per stage: av_prep (sensor, eps per node, q) and av_rhs (LF + viscous RHS + update).  Both
// stage TE elements per block with one thread per node; the FP64 reference matrices sit in shared memory.
#include <cuda_fp16.h>

#include <algorithm>
#include <cstdint>

#include "dg_kernels.cuh"
#include "kernels.hpp"
#include "runner.hpp"

namespace dgk {

namespace {

constexpr int kHid = 32;

__host__ __device__ constexpr int mlp_params(int nin) { return kHid * nin + kHid + kHid * kHid + kHid + kHid + 1; }

template <int N>
struct AvCfg {
  using O = Order<N>;
  static constexpr int NP = O::NP, NFP = O::NFP, NF = O::NF;
  static constexpr int TE = (N <= 2) ? 16 : 8;
  static constexpr int THREADS = ((TE * NP + 31) / 32) * 32;
};

__device__ __forceinline__ double pp_sigma(double S, double s0, double kappa) {
  if (!(S >= s0 - kappa)) return 0.0;
  if (S > s0 + kappa) return 1.0;
  return 0.5 * (1.0 + sin(3.141592653589793 * (S - s0) / (2.0 * kappa)));
}

template <int N>
__global__ void __launch_bounds__(AvCfg<N>::THREADS) av_prep_kernel(const AvArgs A) {
  using C = AvCfg<N>;
  constexpr int NP = C::NP, NFP = C::NFP, NF = C::NF, TE = C::TE;
  extern __shared__ __align__(16) unsigned char sm[];
  double *sDr = reinterpret_cast<double *>(sm);
  double *sDs = sDr + NP * NP, *sDt = sDs + NP * NP, *sVi = sDt + NP * NP, *sL = sVi + NP * NP;
  double *su = sL + NP * NF;          // [TE][NP]
  double *suh = su + TE * NP;         // [TE][NP] modal coefficients, then features
  double *sfl = suh + TE * NP;        // [3][TE][NF]
  double *sfmax = sfl + 3 * TE * NF;  // [TE] feature scale
  double *ssig = sfmax + TE;          // [TE]
  float *sh1 = reinterpret_cast<float *>(ssig + TE);  // [TE][32]
  float *sh2 = sh1 + TE * kHid;                       // [TE][32]
  __half *sW = reinterpret_cast<__half *>(sh2 + TE * kHid);
  int *sfm = reinterpret_cast<int *>(sW + ((mlp_params(NP) + 7) & ~7));
  const int tid = threadIdx.x;
  for (int x = tid; x < NP * NP; x += blockDim.x) {
    sDr[x] = A.Dr[x];
    sDs[x] = A.Ds[x];
    sDt[x] = A.Dt[x];
    sVi[x] = A.Vinv[x];
  }
  for (int x = tid; x < NP * NF; x += blockDim.x) sL[x] = A.LIFT[x];
  for (int x = tid; x < NF; x += blockDim.x) sfm[x] = A.fmask[x];
  if (A.mode == 2)
    for (int x = tid; x < mlp_params(NP); x += blockDim.x) sW[x] = __ushort_as_half(A.mlp16[x]);
  __syncthreads();
  const int e = tid / NP, i = tid - e * NP;
  for (int t = blockIdx.x; t < A.ntiles; t += gridDim.x) {
    const AvTile tl = A.tiles[t];
    const bool act = tid < TE * NP && e < tl.nelem;
    const int64_t nb = tl.node_base + (int64_t)e * NP, fb = tl.face_base + (int64_t)e * NF;
    if (act) su[e * NP + i] = A.u[nb + i];
    __syncthreads();
    if (act) {
      for (int m = i; m < NF; m += NP) {
        const int32_t g = A.gmap[fb + m];
        double uP;
        if ((uint64_t)g < (uint64_t)A.n_u_values) {
          uP = A.u[g];
        } else {
          uP = su[e * NP + sfm[m]];
          atomicExch(A.status, kStatusBadGather);
        }
        const double fs = A.face[3][fb + m];
        const double jump = 0.5 * (uP - su[e * NP + sfm[m]]) * fs;
        for (int d = 0; d < 3; ++d) sfl[(d * TE + e) * NF + m] = A.face[d][fb + m] * jump;
      }
    }
    __syncthreads();
    if (act) {
      const double *ue = su + e * NP;
      double uh = 0.0, ur = 0.0, us = 0.0, ut = 0.0;
#pragma unroll 5
      for (int j = 0; j < NP; ++j) {
        const double v = ue[j];
        uh = fma(sVi[i * NP + j], v, uh);
        ur = fma(sDr[i * NP + j], v, ur);
        us = fma(sDs[i * NP + j], v, us);
        ut = fma(sDt[i * NP + j], v, ut);
      }
      suh[e * NP + i] = uh;
      for (int d = 0; d < 3; ++d) {
        double q = A.geo[d][nb + i] * ur + A.geo[3 + d][nb + i] * us + A.geo[6 + d][nb + i] * ut;
        const double *fl = sfl + (d * TE + e) * NF;
#pragma unroll 6
        for (int m = 0; m < NF; ++m) q = fma(sL[i * NF + m], fl[m], q);
        A.q[d][nb + i] = q;
      }
    }
    __syncthreads();
    // sensor: energy ratio, features, PP activation
    if (act && i == 0) {
      double tot = 0.0, hi = 0.0;
#pragma unroll 5
      for (int j = 0; j < NP; ++j) {
        const double v = suh[e * NP + j];
        tot += v * v;
        if (A.top[j]) hi += v * v;
      }
      const double S = tot > 0.0 ? log10(hi / tot) : -INFINITY;
      const double pp = pp_sigma(S, A.s0, A.kappa);
      ssig[e] = A.mode == 0 ? 0.0 : pp;  // sensor off: no viscosity
      sfmax[e] = tot > 0.0 ? 1.0 / sqrt(tot) : 0.0;  // feature scale: unit-norm modal coefficients
      if (A.S_out) A.S_out[tl.e1_base + e] = (float)S;
      if (A.sig_out) A.sig_out[tl.e1_base + e] = (float)pp;
    }
    __syncthreads();
    if (act) {
      const double f = suh[e * NP + i] * sfmax[e];
      suh[e * NP + i] = f;
      // FP32 copy for the network, in the flux buffer (dead once q is written)
      reinterpret_cast<float *>(sfl)[e * NP + i] = (float)f;
      if (A.feat_out) A.feat_out[tl.feat_base + (int64_t)e * NP + i] = (float)f;
    }
    __syncthreads();
    if (A.mode == 2) {
      // MLP on the unit-norm modal coefficients: FP16 weights, FP32 sums
      const __half *W1 = sW, *b1 = W1 + kHid * NP, *W2 = b1 + kHid, *b2 = W2 + kHid * kHid, *w3 = b2 + kHid,
                   *b3 = w3 + kHid;
      if (act)
        for (int o = i; o < kHid; o += NP) {
          // FP16 weights, FP32 sums in two chains over the FP32 features
          const float *x = reinterpret_cast<const float *>(sfl) + e * NP;
          float s0 = __half2float(b1[o]), s1 = 0.f;
#pragma unroll
          for (int j = 0; j + 1 < NP; j += 2) {
            s0 = fmaf(__half2float(W1[o * NP + j]), x[j], s0);
            s1 = fmaf(__half2float(W1[o * NP + j + 1]), x[j + 1], s1);
          }
          if (NP & 1) s0 = fmaf(__half2float(W1[o * NP + NP - 1]), x[NP - 1], s0);
          sh1[e * kHid + o] = tanhf(s0 + s1);
        }
      __syncthreads();
      if (act)
        for (int o = i; o < kHid; o += NP) {
          float s0 = __half2float(b2[o]), s1 = 0.f;
#pragma unroll
          for (int j = 0; j < kHid; j += 2) {
            s0 = fmaf(__half2float(W2[o * kHid + j]), sh1[e * kHid + j], s0);
            s1 = fmaf(__half2float(W2[o * kHid + j + 1]), sh1[e * kHid + j + 1], s1);
          }
          sh2[e * kHid + o] = tanhf(s0 + s1);
        }
      __syncthreads();
      if (act && i == 0) {
        float z = __half2float(b3[0]);
        for (int j = 0; j < kHid; ++j) z = fmaf(__half2float(w3[j]), sh2[e * kHid + j], z);
        const float sg = 1.f / (1.f + expf(-z));
        if (!(sg > A.conf_lo && sg < A.conf_hi)) {
          ssig[e] = sg;
        } else if (A.fallback_count) {
          atomicAdd(A.fallback_count, 1u);
        }
        if (A.mlp_out) A.mlp_out[tl.e1_base + e] = sg;
      }
      __syncthreads();
    }
    if (act) A.eps[nb + i] = A.eps0 * ssig[e] * A.h_over_n[tl.elem_base + e];
    __syncthreads();
  }
}

template <int N>
__global__ void __launch_bounds__(AvCfg<N>::THREADS) av_rhs_kernel(const AvArgs A) {
  using C = AvCfg<N>;
  constexpr int NP = C::NP, NFP = C::NFP, NF = C::NF, TE = C::TE;
  extern __shared__ __align__(16) unsigned char sm[];
  double *sDr = reinterpret_cast<double *>(sm);
  double *sDs = sDr + NP * NP, *sDt = sDs + NP * NP, *sL = sDt + NP * NP;
  double *su = sL + NP * NF;    // [TE][NP]
  double *sq = su + TE * NP;    // [3][TE][NP]
  double *sfl = sq + 3 * TE * NP;  // [TE][NF]
  int *sfm = reinterpret_cast<int *>(sfl + TE * NF);
  const int tid = threadIdx.x;
  for (int x = tid; x < NP * NP; x += blockDim.x) {
    sDr[x] = A.Dr[x];
    sDs[x] = A.Ds[x];
    sDt[x] = A.Dt[x];
  }
  for (int x = tid; x < NP * NF; x += blockDim.x) sL[x] = A.LIFT[x];
  for (int x = tid; x < NF; x += blockDim.x) sfm[x] = A.fmask[x];
  __syncthreads();
  const int e = tid / NP, i = tid - e * NP;
  const double a = A.a, b = A.b, dt = A.dt;
  for (int t = blockIdx.x; t < A.ntiles; t += gridDim.x) {
    const AvTile tl = A.tiles[t];
    const bool act = tid < TE * NP && e < tl.nelem;
    const int64_t nb = tl.node_base + (int64_t)e * NP, fb = tl.face_base + (int64_t)e * NF;
    if (act) {
      su[e * NP + i] = A.u[nb + i];
      for (int d = 0; d < 3; ++d) sq[(d * TE + e) * NP + i] = A.q[d][nb + i];
    }
    __syncthreads();
    if (act) {
      const double epsM = A.eps[nb];  // constant per element
      for (int m = i; m < NF; m += NP) {
        const int32_t g = A.gmap[fb + m];
        const int jM = sfm[m];
        const double uM = su[e * NP + jM];
        double uP, eP, qP[3];
        if ((uint64_t)g < (uint64_t)A.n_u_values) {
          uP = A.u[g];
          eP = A.eps[g];
          for (int d = 0; d < 3; ++d) qP[d] = A.q[d][g];
        } else {
          uP = uM;
          eP = epsM;
          for (int d = 0; d < 3; ++d) qP[d] = sq[(d * TE + e) * NP + jM];
          atomicExch(A.status, kStatusBadGather);
        }
        const double nx = A.face[0][fb + m], ny = A.face[1][fb + m], nz = A.face[2][fb + m];
        const double fs = A.face[3][fb + m];
        const double ns = nx + ny + nz;
        const double fM = 0.5 * uM * uM * ns, fP = 0.5 * uP * uP * ns;
        const double C = fmax(fabs(uM) * fabs(ns), fabs(uP) * fabs(ns));
        const double du = fM - (0.5 * (fM + fP) + 0.5 * C * (uM - uP));
        const double nv[3] = {nx, ny, nz};
        double vis = 0.0;
        for (int d = 0; d < 3; ++d) vis += nv[d] * (eP * qP[d] - epsM * sq[(d * TE + e) * NP + jM]);
        sfl[e * NF + m] = fs * du + 0.5 * fs * vis;
      }
    }
    __syncthreads();
    if (act) {
      const double *ue = su + e * NP;
      double ur = 0.0, us = 0.0, ut = 0.0;
#pragma unroll 5
      for (int j = 0; j < NP; ++j) {
        ur = fma(sDr[i * NP + j], ue[j], ur);
        us = fma(sDs[i * NP + j], ue[j], us);
        ut = fma(sDt[i * NP + j], ue[j], ut);
      }
      const double ux = A.geo[0][nb + i] * ur + A.geo[3][nb + i] * us + A.geo[6][nb + i] * ut;
      const double uy = A.geo[1][nb + i] * ur + A.geo[4][nb + i] * us + A.geo[7][nb + i] * ut;
      const double uz = A.geo[2][nb + i] * ur + A.geo[5][nb + i] * us + A.geo[8][nb + i] * ut;
      double rhs = -ue[i] * (ux + uy + uz);
      const double eps = A.eps[nb + i];
      if (eps != 0.0) {
        double div = 0.0;
        for (int d = 0; d < 3; ++d) {
          const double *qd = sq + (d * TE + e) * NP;
          double qr = 0.0, qs = 0.0, qt = 0.0;
    #pragma unroll 5
      for (int j = 0; j < NP; ++j) {
            qr = fma(sDr[i * NP + j], qd[j], qr);
            qs = fma(sDs[i * NP + j], qd[j], qs);
            qt = fma(sDt[i * NP + j], qd[j], qt);
          }
          div += A.geo[d][nb + i] * qr + A.geo[3 + d][nb + i] * qs + A.geo[6 + d][nb + i] * qt;
        }
        rhs += eps * div;
      }
      const double *fl = sfl + e * NF;
      double lift = 0.0;
#pragma unroll 6
      for (int m = 0; m < NF; ++m) lift = fma(sL[i * NF + m], fl[m], lift);
      rhs += lift;
      const double r = a * A.resu[nb + i] + dt * rhs;
      A.resu[nb + i] = r;
      A.u_out[nb + i] = ue[i] + b * r;
    }
    __syncthreads();
  }
}

template <int N>
size_t prep_smem(int np_, int nf_) {
  using C = AvCfg<N>;
  (void)np_;
  (void)nf_;
  constexpr int NP = C::NP, NF = C::NF, TE = C::TE;
  size_t b = sizeof(double) * (4 * NP * NP + NP * NF + 2 * TE * NP + 3 * TE * NF + 2 * TE);
  b += sizeof(float) * 2 * TE * kHid;
  b += sizeof(__half) * ((mlp_params(NP) + 7) & ~7);
  b += sizeof(int) * NF;
  return b;
}

template <int N>
size_t rhs_smem() {
  using C = AvCfg<N>;
  constexpr int NP = C::NP, NF = C::NF, TE = C::TE;
  return sizeof(double) * (3 * NP * NP + NP * NF + 4 * TE * NP + TE * NF) + sizeof(int) * NF;
}

template <int N>
void launch_av_n(const AvArgs &A, int num_sms, cudaStream_t st) {
  using C = AvCfg<N>;
  const size_t s1 = prep_smem<N>(C::NP, C::NF), s2 = rhs_smem<N>();
  cuda_check(cudaFuncSetAttribute(av_prep_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s1),
             "av_prep smem");
  cuda_check(cudaFuncSetAttribute(av_rhs_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s2),
             "av_rhs smem");
  const int grid = std::max(1, std::min(A.ntiles, num_sms * 8));
  av_prep_kernel<N><<<grid, C::THREADS, s1, st>>>(A);
  cuda_check(cudaGetLastError(), "av_prep_kernel launch");
  if (A.prep_only) return;
  av_rhs_kernel<N><<<grid, C::THREADS, s2, st>>>(A);
  cuda_check(cudaGetLastError(), "av_rhs_kernel launch");
}

// ---------------- MLP: forward, loss gradient (mean squared error), Adam, FP32 -> FP16 ----------------

template <int NIN>
__device__ __forceinline__ float mlp_fwd(const float *p, const float *x, float *h1, float *h2) {
  const float *W1 = p, *b1 = W1 + kHid * NIN, *W2 = b1 + kHid, *b2 = W2 + kHid * kHid, *w3 = b2 + kHid,
              *b3 = w3 + kHid;
#pragma unroll 4
  for (int o = 0; o < kHid; ++o) {
    float s = b1[o];
    for (int j = 0; j < NIN; ++j) s = fmaf(W1[o * NIN + j], x[j], s);
    h1[o] = tanhf(s);
  }
#pragma unroll 4
  for (int o = 0; o < kHid; ++o) {
    float s = b2[o];
    for (int j = 0; j < kHid; ++j) s = fmaf(W2[o * kHid + j], h1[j], s);
    h2[o] = tanhf(s);
  }
  float z = b3[0];
  for (int j = 0; j < kHid; ++j) z = fmaf(w3[j], h2[j], z);
  return 1.f / (1.f + expf(-z));
}

template <int NIN>
__global__ void mlp_forward_kernel(const float *p, const float *X, int64_t n, float *out) {
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
    float x[NIN], h1[kHid], h2[kHid];
    for (int j = 0; j < NIN; ++j) x[j] = X[s * NIN + j];
    out[s] = mlp_fwd<NIN>(p, x, h1, h2);
  }
}

// Gradient of mean((mlp(x) - y)^2) over n samples; every block sums its samples' gradients in shared memory
// and adds them to `grad` (zeroed by the caller).  `loss` receives the sum of squared errors / n.
template <int NIN>
__global__ void mlp_grad_kernel(const float *p, const float *X, const float *y, int64_t n, float *grad, float *loss) {
  constexpr int P = mlp_params(NIN);
  extern __shared__ float sg[];  // [P + 1]
  for (int x = threadIdx.x; x <= P; x += blockDim.x) sg[x] = 0.f;
  __syncthreads();
  const float *W2 = p + kHid * NIN + kHid, *w3 = W2 + kHid * kHid + kHid;
  float *gW1 = sg, *gb1 = gW1 + kHid * NIN, *gW2 = gb1 + kHid, *gb2 = gW2 + kHid * kHid, *gw3 = gb2 + kHid,
        *gb3 = gw3 + kHid;
  const float inv_n = 1.f / (float)n;
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
    float x[NIN], h1[kHid], h2[kHid];
    for (int j = 0; j < NIN; ++j) x[j] = X[s * NIN + j];
    const float o = mlp_fwd<NIN>(p, x, h1, h2);
    const float r = o - y[s];
    atomicAdd(&sg[P], r * r * inv_n);
    const float dz = 2.f * r * o * (1.f - o) * inv_n;
    atomicAdd(gb3, dz);
    float d2[kHid];
    for (int j = 0; j < kHid; ++j) {
      atomicAdd(&gw3[j], dz * h2[j]);
      d2[j] = dz * w3[j] * (1.f - h2[j] * h2[j]);
    }
    for (int oo = 0; oo < kHid; ++oo) {
      atomicAdd(&gb2[oo], d2[oo]);
      for (int j = 0; j < kHid; ++j) atomicAdd(&gW2[oo * kHid + j], d2[oo] * h1[j]);
    }
    for (int j = 0; j < kHid; ++j) {
      float s1 = 0.f;
      for (int oo = 0; oo < kHid; ++oo) s1 = fmaf(W2[oo * kHid + j], d2[oo], s1);
      const float d1 = s1 * (1.f - h1[j] * h1[j]);
      atomicAdd(&gb1[j], d1);
      for (int k = 0; k < NIN; ++k) atomicAdd(&gW1[j * NIN + k], d1 * x[k]);
    }
  }
  __syncthreads();
  for (int x = threadIdx.x; x < P; x += blockDim.x)
    if (sg[x] != 0.f) atomicAdd(&grad[x], sg[x]);
  if (threadIdx.x == 0) atomicAdd(loss, sg[P]);
}

__global__ void adam_kernel(float *p, const float *g, float *m, float *v, int64_t P, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < P; k += (int64_t)gridDim.x * blockDim.x) {
    const float gk = g[k];
    const float mk = b1 * m[k] + (1.f - b1) * gk;
    const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    p[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
  }
}

__global__ void to_half_kernel(const float *in, __half *out, int64_t n) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    out[k] = __float2half_rn(in[k]);
}

// FP16-weight forward, the arithmetic of the sensor kernel: weights rounded to FP16, sums in FP32.
template <int NIN>
__global__ void mlp_forward16_kernel(const __half *p, const float *X, int64_t n, float *out) {
  constexpr int P = mlp_params(NIN);
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
    const __half *W1 = p, *b1 = W1 + kHid * NIN, *W2 = b1 + kHid, *b2 = W2 + kHid * kHid, *w3 = b2 + kHid,
                 *b3 = w3 + kHid;
    (void)P;
    float h1[kHid], h2[kHid];
    for (int o = 0; o < kHid; ++o) {
      float sum = __half2float(b1[o]);
      for (int j = 0; j < NIN; ++j) sum = fmaf(__half2float(W1[o * NIN + j]), X[s * NIN + j], sum);
      h1[o] = tanhf(sum);
    }
    for (int o = 0; o < kHid; ++o) {
      float sum = __half2float(b2[o]);
      for (int j = 0; j < kHid; ++j) sum = fmaf(__half2float(W2[o * kHid + j]), h1[j], sum);
      h2[o] = tanhf(sum);
    }
    float z = __half2float(b3[0]);
    for (int j = 0; j < kHid; ++j) z = fmaf(__half2float(w3[j]), h2[j], z);
    out[s] = 1.f / (1.f + expf(-z));
  }
}

}  // namespace

int mlp_param_count(int nin) { return mlp_params(nin); }

int av_tile_elems(int N) { return N <= 2 ? AvCfg<2>::TE : AvCfg<3>::TE; }

void launch_av(int N, const AvArgs &A, int num_sms, cudaStream_t st) {
  switch (N) {
    case 1: launch_av_n<1>(A, num_sms, st); break;
    case 2: launch_av_n<2>(A, num_sms, st); break;
    case 3: launch_av_n<3>(A, num_sms, st); break;
    case 4: launch_av_n<4>(A, num_sms, st); break;
    case 5: launch_av_n<5>(A, num_sms, st); break;
    default: throw Error(DGK_ERR_UNSUPPORTED, "artificial-viscosity stage: orders 1..5");
  }
}

void launch_to_half(const float *in, void *out, int64_t n, cudaStream_t st) {
  to_half_kernel<<<std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 4096)), 256, 0, st>>>(
      in, reinterpret_cast<__half *>(out), n);
  cuda_check(cudaGetLastError(), "to_half_kernel launch");
}

#define DGK_NIN_SWITCH(nin, CALL)                                                     \
  switch (nin) {                                                                      \
    case 4: CALL(4); break;                                                           \
    case 10: CALL(10); break;                                                         \
    case 20: CALL(20); break;                                                         \
    case 35: CALL(35); break;                                                         \
    case 56: CALL(56); break;                                                         \
    default: throw Error(DGK_ERR_UNSUPPORTED, "MLP input width must be Np of order 1..5"); \
  }

void launch_mlp_forward(const float *p, const float *X, int64_t n, int nin, float *out, int fp16, void *half_buf,
                        cudaStream_t st) {
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((n + 127) / 128, 8192));
  if (fp16) {
    launch_to_half(p, half_buf, mlp_params(nin), st);
#define F16(NIN) mlp_forward16_kernel<NIN><<<blocks, 128, 0, st>>>(reinterpret_cast<const __half *>(half_buf), X, n, out)
    DGK_NIN_SWITCH(nin, F16)
#undef F16
  } else {
#define F32(NIN) mlp_forward_kernel<NIN><<<blocks, 128, 0, st>>>(p, X, n, out)
    DGK_NIN_SWITCH(nin, F32)
#undef F32
  }
  cuda_check(cudaGetLastError(), "mlp forward launch");
}

void launch_mlp_grad(const float *p, const float *X, const float *y, int64_t n, int nin, float *grad, float *loss,
                     cudaStream_t st) {
  const int P = mlp_params(nin);
  cuda_check(cudaMemsetAsync(grad, 0, sizeof(float) * P, st), "zero grad");
  cuda_check(cudaMemsetAsync(loss, 0, sizeof(float), st), "zero loss");
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 1184));
  const size_t sm = sizeof(float) * (P + 1);
#define G(NIN) mlp_grad_kernel<NIN><<<blocks, 256, sm, st>>>(p, X, y, n, grad, loss)
  DGK_NIN_SWITCH(nin, G)
#undef G
  cuda_check(cudaGetLastError(), "mlp grad launch");
}

void launch_adam(float *p, const float *g, float *m, float *v, int64_t P, float lr, float b1, float b2, float eps,
                 int step, cudaStream_t st) {
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  adam_kernel<<<std::max<int64_t>(1, std::min<int64_t>((P + 255) / 256, 1024)), 256, 0, st>>>(p, g, m, v, P, lr, b1,
                                                                                                b2, eps, c1, c2);
  cuda_check(cudaGetLastError(), "adam launch");
}

}  // namespace dgk
