// sm_100a kernels: type conversion for the copy engine, and the tet-DG hot path (volume derivative,
// reference-form computeRHS / updateSolution, fused Lax-Friedrichs RHS + LSERK4 stage).
#include <cstdint>
#include <type_traits>

#include "dg_kernels.cuh"
#include "kernels.hpp"
#include "runner.hpp"

namespace dgk {

// ------------------------------------------------------------------------------------------------
// copy engine: dtype conversion and mat.Matrix transposes (runner/memory_operations.go:243-418,
// runner/kernel_copy.go:86-140)
// ------------------------------------------------------------------------------------------------
template <typename S, typename D>
__global__ void convert_kernel(const S *__restrict__ s, D *__restrict__ d, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    d[i] = (D)s[i];
}

// to_cm: s is row-major rows x cols, d column-major (d[c*rows + r] = s[r*cols + c]); else the inverse.
template <typename S, typename D>
__global__ void transpose_kernel(const S *__restrict__ s, D *__restrict__ d, int64_t rows, int64_t cols, bool to_cm) {
  __shared__ D tile[32][33];
  const int64_t r0 = (int64_t)blockIdx.y * 32, c0 = (int64_t)blockIdx.x * 32;
  // read a 32x32 block coalesced along the source's contiguous dimension
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int64_t r = r0 + k, c = c0 + threadIdx.x;
    if (to_cm) {
      if (r < rows && c < cols) tile[k][threadIdx.x] = (D)s[r * cols + c];
    } else {
      // source column-major: element (r', c') at c' * rows + r'; walk rows along x
      const int64_t rr = r0 + threadIdx.x, cc = c0 + k;
      if (rr < rows && cc < cols) tile[threadIdx.x][k] = (D)s[cc * rows + rr];
    }
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    if (to_cm) {
      const int64_t c = c0 + k, r = r0 + threadIdx.x;
      if (r < rows && c < cols) d[c * rows + r] = tile[threadIdx.x][k];
    } else {
      const int64_t r = r0 + k, c = c0 + threadIdx.x;
      if (r < rows && c < cols) d[r * cols + c] = tile[k][threadIdx.x];
    }
  }
}

template <typename F>
static void by_type(int dt, F &&f) {
  switch (dt) {
    case DGK_FLOAT32: f(float{}); break;
    case DGK_FLOAT64: f(double{}); break;
    case DGK_INT32: f(int32_t{}); break;
    case DGK_INT64: f(int64_t{}); break;
    default: throw Error(DGK_ERR_INVALID, "bad dtype");
  }
}

void launch_convert(const void *src, int sdt, void *dst, int ddt, int64_t n, cudaStream_t st) {
  if (n <= 0) return;
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
  by_type(sdt, [&](auto s) {
    by_type(ddt, [&](auto d) {
      using S = decltype(s);
      using D = decltype(d);
      convert_kernel<S, D><<<blocks, 256, 0, st>>>(static_cast<const S *>(src), static_cast<D *>(dst), n);
    });
  });
}

void launch_transpose_convert(const void *src, int sdt, void *dst, int ddt, int64_t rows, int64_t cols, bool to_cm,
                              cudaStream_t st) {
  if (rows <= 0 || cols <= 0) return;
  dim3 grid((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32)), block(32, 8);
  if (grid.y > 65535) throw Error(DGK_ERR_UNSUPPORTED, "matrix too tall for the transpose kernel");
  by_type(sdt, [&](auto s) {
    by_type(ddt, [&](auto d) {
      using S = decltype(s);
      using D = decltype(d);
      transpose_kernel<S, D><<<grid, block, 0, st>>>(static_cast<const S *>(src), static_cast<D *>(dst), rows, cols,
                                                     to_cm);
    });
  });
}

// ------------------------------------------------------------------------------------------------
// hot path
// ------------------------------------------------------------------------------------------------
// Streaming loads/stores for data touched once per stage (metrics, face data, residual): evict-first so
// L2 keeps the state array whose neighbour traces the face gather re-reads.
template <typename T>
__device__ __forceinline__ T lds(const T *p) { return __ldcs(p); }
template <typename T>
__device__ __forceinline__ void sts(T *p, T v) { __stcs(p, v); }

// Bulk prefetch of a contiguous global range into L2 (TMA, no shared memory involved).  The range is widened
// to 16-byte granules; every array lives in a 256-byte aligned slot of the runner's arena, so the widened
// range stays inside the array's slot.
__device__ __forceinline__ void prefetch_l2(const void *p, size_t bytes) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(p) & ~uintptr_t(15);
  const uintptr_t e = (reinterpret_cast<uintptr_t>(p) + bytes + 15) & ~uintptr_t(15);
  if (e > a) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((unsigned)(e - a)) : "memory");
}

// Row stride of a matrix staged in shared memory: even, so (j, j+1) pairs load as one 16-byte vector.
template <int C>
struct Pad {
  static constexpr int V = (C + 1) & ~1;
};

// NM stacked NR x NC matrices (row stride Pad<NC>::V) times one element vector of a shared-memory tile, for
// the RG rows of row group g: acc[m][r] = sum_j M[m][g*RG + r][j] * f(x[j]), f(x) = x or x^2/2.  The j loop
// walks column pairs so each matrix entry pair is one 128-bit broadcast load.
template <typename T, int NR, int NC, int RG, int NM, bool SQUARE>
__device__ __forceinline__ void rows_matvec(const T *__restrict__ M, const T *xe, int g, T (&acc)[NM][RG]) {
  constexpr int LD = Pad<NC>::V;
  using T2 = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
#pragma unroll
  for (int m = 0; m < NM; ++m)
#pragma unroll
    for (int r = 0; r < RG; ++r) acc[m][r] = T(0);
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
#pragma unroll
      for (int m = 0; m < NM; ++m) {
        const T2 mm = *reinterpret_cast<const T2 *>(M + (m * NR + i) * LD + j);
        acc[m][r] = fma(mm.x, x0, acc[m][r]);
        acc[m][r] = fma(mm.y, x1, acc[m][r]);
      }
    }
  }
  if (NC & 1) {
    T x0 = xe[NC - 1];
    if (SQUARE) x0 = T(0.5) * x0 * x0;
#pragma unroll
    for (int r = 0; r < RG; ++r) {
      const int i = min(i0 + r, NR - 1);
#pragma unroll
      for (int m = 0; m < NM; ++m) acc[m][r] = fma(M[(m * NR + i) * LD + NC - 1], x0, acc[m][r]);
    }
  }
}

// Issue L2 prefetches for every stream a tile of the fused stage reads.
template <typename T>
__device__ __forceinline__ void prefetch_tile(const RhsArgs<T> &A, const Tile &tl, int np, int nf) {
  const size_t nn = (size_t)tl.nelem * np, fn = (size_t)tl.nelem * nf;
  prefetch_l2(A.u_in + tl.node_base, nn * sizeof(T));
  if (A.resu) prefetch_l2(A.resu + tl.node_base, nn * sizeof(T));
#pragma unroll
  for (int k = 0; k < 9; ++k) prefetch_l2(A.geo[k] + tl.node_base, nn * sizeof(T));
#pragma unroll
  for (int k = 0; k < 4; ++k) prefetch_l2(A.face[k] + tl.face_base, fn * sizeof(T));
  prefetch_l2(A.gmap + tl.face_base, fn * sizeof(int32_t));
}

// Shared-memory carve-up of the fused kernels.
template <typename T, int N, bool MSMEM>
struct Smem {
  using O = Order<N>;
  using C = Cfg<N>;
  static constexpr int DM = MSMEM ? 3 * O::NP * Pad<O::NP>::V : 0;
  static constexpr int LM = MSMEM ? O::NP * Pad<O::NF>::V : 0;
  static constexpr int U = C::TE * O::NPS;
  static constexpr int D3 = 3 * C::TE * O::NPS;
  static constexpr int F = C::TE * O::NFS;
  static constexpr size_t bytes = sizeof(T) * (size_t)(DM + LM + U + D3 + F) + sizeof(int) * O::NF;
};

template <typename T, int N, bool MSMEM>
__global__ void __launch_bounds__(Cfg<N>::THREADS, 2) rhs_stage_kernel(RhsArgs<T> A, int rhs_only) {
  using O = Order<N>;
  using C = Cfg<N>;
  using S = Smem<T, N, MSMEM>;
  constexpr int NP = O::NP, NF = O::NF, NPS = O::NPS, NFS = O::NFS, TE = C::TE, RG = C::RG;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sD = reinterpret_cast<T *>(smem_raw);
  T *sL = sD + S::DM;
  T *su = sL + S::LM;
  T *sd = su + S::U;
  T *sf = sd + S::D3;
  int *sfm = reinterpret_cast<int *>(sf + S::F);
  const int tid = threadIdx.x, nth = C::THREADS;  // launched with exactly Cfg<N>::THREADS threads
  if (tid == 0 && blockIdx.x < A.ntiles) prefetch_tile(A, A.tiles[blockIdx.x], NP, NF);
  if (MSMEM) {  // the operator stores both matrices with the padded row strides used here
    for (int i = tid; i < S::DM; i += nth) sD[i] = A.Dmat[i];
    for (int i = tid; i < S::LM; i += nth) sL[i] = A.LIFT[i];
  }
  for (int i = tid; i < NF; i += nth) sfm[i] = A.fmask[i];
  const T *Dm = MSMEM ? sD : A.Dmat;
  const T *Lm = MSMEM ? sL : A.LIFT;
  const int e_own = tid % TE, g_own = tid / TE;
  const T a = A.a, b = A.b, dt = A.dt;
  __syncthreads();

  // Per-thread item counts of the element-contiguous (flat) phases.  Each flat phase issues the loads of a
  // whole batch before consuming any, so a tile costs a few memory round trips per phase instead of one per
  // item; batch sizes keep the loaded values within a modest register budget.
  constexpr int THREADS = C::THREADS;
  constexpr int NI = (TE * NP + THREADS - 1) / THREADS;  // node items per thread
  constexpr int NJ = (TE * NF + THREADS - 1) / THREADS;  // face items per thread
  constexpr int WORDS = sizeof(T) / 4;                    // 32-bit registers per value
  constexpr int CHN = (54 / (9 * WORDS)) > 0 ? (54 / (9 * WORDS)) : 1;  // metric batch (9 values per item)
  constexpr int CHF = (40 / (4 * WORDS)) > 0 ? (40 / (4 * WORDS)) : 1;  // face-data batch (4 values per item)

  for (int t = blockIdx.x; t < A.ntiles; t += gridDim.x) {
    const Tile tl = A.tiles[t];
    if (tid == 0 && t + (int)gridDim.x < A.ntiles) prefetch_tile(A, A.tiles[t + gridDim.x], NP, NF);
    const int ne = tl.nelem, nn = ne * NP, nfc = ne * NF;
    const T *ug = A.u_in + tl.node_base;
    // P0: the tile's state, coalesced
    {
      T v[NI];
#pragma unroll
      for (int k = 0; k < NI; ++k) {
        const int idx = tid + k * THREADS;
        v[k] = idx < nn ? ug[idx] : T(0);
      }
#pragma unroll
      for (int k = 0; k < NI; ++k) {
        const int idx = tid + k * THREADS;
        if (idx < nn) {
          const int e = idx / NP, i = idx - e * NP;
          su[e * NPS + i] = v[k];
        }
      }
    }
    // P0b: neighbour traces uP through the fused exchange map into the flux buffer (index batch, then gather batch)
    {
      int32_t src[NJ];
#pragma unroll
      for (int k = 0; k < NJ; ++k) {
        const int idx = tid + k * THREADS;
        src[k] = idx < nfc ? lds(A.gmap + tl.face_base + idx) : 0;
      }
      T up[NJ];
#pragma unroll
      for (int k = 0; k < NJ; ++k) {
        const int idx = tid + k * THREADS;
        const bool ok = src[k] >= 0 && (int64_t)src[k] < A.n_u_values;
        up[k] = (idx < nfc && ok) ? A.u_in[src[k]] : T(0);
        if (idx < nfc && !ok) atomicExch(A.status, kStatusBadGather);
      }
#pragma unroll
      for (int k = 0; k < NJ; ++k) {
        const int idx = tid + k * THREADS;
        if (idx < nfc) {
          const int e = idx / NF, q = idx - e * NF;
          const bool ok = src[k] >= 0 && (int64_t)src[k] < A.n_u_values;
          // a rejected index (reported above) falls back to the interior trace uM
          sf[e * NFS + q] = ok ? up[k] : A.u_in[tl.node_base + e * NP + sfm[q]];
        }
      }
    }
    __syncthreads();
    // P1: ur, us, ut (of u, or of u^2/2 in conservative form) for this thread's element and rows
    if (e_own < ne) {
      // one derivative matrix at a time keeps a single accumulator set live
#pragma unroll 1
      for (int m = 0; m < 3; ++m) {
        T acc[1][RG];
        if (A.conservative)
          rows_matvec<T, NP, NP, RG, 1, true>(Dm + m * NP * Pad<NP>::V, su + e_own * NPS, g_own, acc);
        else
          rows_matvec<T, NP, NP, RG, 1, false>(Dm + m * NP * Pad<NP>::V, su + e_own * NPS, g_own, acc);
#pragma unroll
        for (int r = 0; r < RG; ++r) {
          const int i = g_own * RG + r;
          if (i < NP) sd[m * TE * NPS + e_own * NPS + i] = acc[0][r];
        }
      }
    }
    __syncthreads();
    // P2a: volume term with the per-node metrics (coalesced streams, CHN items per batch)
#pragma unroll
    for (int k0 = 0; k0 < NI; k0 += CHN) {
      T gm[CHN][9];
#pragma unroll
      for (int k = 0; k < CHN; ++k) {
        const int idx = tid + (k0 + k) * THREADS;
        if (k0 + k < NI && idx < nn) {
#pragma unroll
          for (int m = 0; m < 9; ++m) gm[k][m] = lds(A.geo[m] + tl.node_base + idx);
        }
      }
#pragma unroll
      for (int k = 0; k < CHN; ++k) {
        const int idx = tid + (k0 + k) * THREADS;
        if (k0 + k < NI && idx < nn) {
          const int e = idx / NP, i = idx - e * NP;
          const int so = e * NPS + i;
          const T ur = sd[so], us = sd[TE * NPS + so], ut = sd[2 * TE * NPS + so];
          const T ux = gm[k][0] * ur + gm[k][3] * us + gm[k][6] * ut;
          const T uy = gm[k][1] * ur + gm[k][4] * us + gm[k][7] * ut;
          const T uz = gm[k][2] * ur + gm[k][5] * us + gm[k][8] * ut;
          sd[so] = A.conservative ? -(ux + uy + uz) : -su[so] * (ux + uy + uz);
        }
      }
    }
    // P2b: Lax-Friedrichs surface term at every face point (face data in CHF-item batches)
#pragma unroll
    for (int k0 = 0; k0 < NJ; k0 += CHF) {
      T fc[CHF][4];
#pragma unroll
      for (int k = 0; k < CHF; ++k) {
        const int idx = tid + (k0 + k) * THREADS;
        if (k0 + k < NJ && idx < nfc) {
#pragma unroll
          for (int m = 0; m < 4; ++m) fc[k][m] = lds(A.face[m] + tl.face_base + idx);
        }
      }
#pragma unroll
      for (int k = 0; k < CHF; ++k) {
        const int idx = tid + (k0 + k) * THREADS;
        if (k0 + k < NJ && idx < nfc) {
          const int e = idx / NF, q = idx - e * NF;
          const T uM = su[e * NPS + sfm[q]];
          const T uP = sf[e * NFS + q];
          const T nsum = fc[k][0] + fc[k][1] + fc[k][2];
          const T fM = T(0.5) * uM * uM * nsum, fP = T(0.5) * uP * uP * nsum;
          const T an = fabs(nsum);
          const T lam = fmax(fabs(uM) * an, fabs(uP) * an);
          const T du = fM - (T(0.5) * (fM + fP) + T(0.5) * lam * (uM - uP));
          sf[e * NFS + q] = fc[k][3] * du;
        }
      }
    }
    __syncthreads();
    // P3: rhs = volume + LIFT * (Fscale du)
    if (e_own < ne) {
      T acc[1][RG];
      rows_matvec<T, NP, NF, RG, 1, false>(Lm, sf + e_own * NFS, g_own, acc);
#pragma unroll
      for (int r = 0; r < RG; ++r) {
        const int i = g_own * RG + r;
        if (i < NP) sd[e_own * NPS + i] += acc[0][r];
      }
    }
    __syncthreads();
    // P4: LSERK4 stage (or the bare RHS), coalesced
    {
      T rs[NI];
#pragma unroll
      for (int k = 0; k < NI; ++k) {
        const int idx = tid + k * THREADS;
        rs[k] = (!rhs_only && idx < nn) ? lds(A.resu + tl.node_base + idx) : T(0);
      }
#pragma unroll
      for (int k = 0; k < NI; ++k) {
        const int idx = tid + k * THREADS;
        if (idx < nn) {
          const int e = idx / NP, i = idx - e * NP;
          const int64_t gi = tl.node_base + idx;
          const T rhs = sd[e * NPS + i];
          if (rhs_only) {
            sts(A.rhs_out + gi, rhs);
          } else {
            const T res = a * rs[k] + dt * rhs;
            sts(A.resu + gi, res);
            sts(A.u_out + gi, su[e * NPS + i] + b * res);
          }
        }
      }
    }
    __syncthreads();
  }
}

// Volume derivative microbench (`differentiate`) and the reference's volume-only computeRHS.
template <typename T, int N, bool MSMEM>
__global__ void __launch_bounds__(Cfg<N>::THREADS) diff_kernel(DiffArgs<T> A) {
  using O = Order<N>;
  using C = Cfg<N>;
  constexpr int NP = O::NP, NPS = O::NPS, TE = C::TE, RG = C::RG;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sD = reinterpret_cast<T *>(smem_raw);
  T *su = sD + (MSMEM ? 3 * NP * Pad<NP>::V : 0);
  T *sd = su + TE * NPS;
  const int tid = threadIdx.x, nth = blockDim.x;
  if (MSMEM)
    for (int i = tid; i < 3 * NP * Pad<NP>::V; i += nth) sD[i] = A.Dmat[i];
  const T *Dm = MSMEM ? sD : A.Dmat;
  const int e_own = tid % TE, g_own = tid / TE;
  __syncthreads();
  for (int t = blockIdx.x; t < A.ntiles; t += gridDim.x) {
    const Tile tl = A.tiles[t];
    const int ne = tl.nelem;
    for (int idx = tid; idx < ne * NP; idx += nth) {
      const int e = idx / NP, i = idx - e * NP;
      su[e * NPS + i] = lds(A.u + tl.node_base + idx);
    }
    __syncthreads();
    if (e_own < ne) {
      T acc[3][RG];
      rows_matvec<T, NP, NP, RG, 3, false>(Dm, su + e_own * NPS, g_own, acc);
#pragma unroll
      for (int r = 0; r < RG; ++r) {
        const int i = g_own * RG + r;
        if (i < NP) {
#pragma unroll
          for (int m = 0; m < 3; ++m) sd[m * TE * NPS + e_own * NPS + i] = acc[m][r];
        }
      }
    }
    __syncthreads();
    for (int idx = tid; idx < ne * NP; idx += nth) {
      const int e = idx / NP, i = idx - e * NP;
      const int64_t gi = tl.node_base + idx;
      const int so = e * NPS + i;
      const T ur = sd[so], us = sd[TE * NPS + so], ut = sd[2 * TE * NPS + so];
      const T ux = lds(A.geo[0] + gi) * ur + lds(A.geo[3] + gi) * us + lds(A.geo[6] + gi) * ut;
      const T uy = lds(A.geo[1] + gi) * ur + lds(A.geo[4] + gi) * us + lds(A.geo[7] + gi) * ut;
      const T uz = lds(A.geo[2] + gi) * ur + lds(A.geo[5] + gi) * us + lds(A.geo[8] + gi) * ut;
      if (A.mode == 0) {
        sts(A.out[0] + gi, ux);
        sts(A.out[1] + gi, uy);
        sts(A.out[2] + gi, uz);
      } else {
        sts(A.out[0] + gi, -su[so] * (ux + uy + uz));
      }
    }
    __syncthreads();
  }
}

// Elementwise updates over tiles: mode 0 = the reference's updateSolution
// (resu = rka*resu + rkb*rhsu; u += resu), mode 1 = standard LSERK4 (resu = a*resu + dt*rhs; u += b*resu).
template <typename T>
__global__ void update_kernel(const Tile *tiles, int ntiles, int np, T *u, T *resu, const T *rhs, T c0, T c1, T c2,
                              int mode) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const int n = tl.nelem * np;
    for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
      const int64_t gi = tl.node_base + idx;
      if (mode == 0) {
        const T r = c0 * resu[gi] + c1 * rhs[gi];
        resu[gi] = r;
        u[gi] = u[gi] + r;
      } else {
        const T r = c0 * resu[gi] + c2 * rhs[gi];
        resu[gi] = r;
        u[gi] = u[gi] + c1 * r;
      }
    }
  }
}

// ------------------------------------------------------------------------------------------------
// host launchers
// ------------------------------------------------------------------------------------------------
template <typename T, int N>
static bool mats_fit() {
  return Smem<T, N, true>::bytes <= 200 * 1024;
}

template <typename K>
static int resident(K kernel, int threads, size_t smem) {
  cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attr");
  int n = 0;
  cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem), "occupancy");
  return n;
}

template <typename T, int N>
static void rhs_launch_n(const RhsArgs<T> &A, int rhs_only, int num_sms, cudaStream_t st, LaunchInfo *info) {
  const int threads = Cfg<N>::THREADS;
  if (mats_fit<T, N>()) {
    auto k = rhs_stage_kernel<T, N, true>;
    const size_t sm = Smem<T, N, true>::bytes;
    const int per = std::max(1, resident(k, threads, sm));
    const int grid = std::min(A.ntiles, per * num_sms);
    if (info) *info = {grid, threads, (int)sm, per};
    if (grid > 0) k<<<grid, threads, sm, st>>>(A, rhs_only);
  } else {
    auto k = rhs_stage_kernel<T, N, false>;
    const size_t sm = Smem<T, N, false>::bytes;
    const int per = std::max(1, resident(k, threads, sm));
    const int grid = std::min(A.ntiles, per * num_sms);
    if (info) *info = {grid, threads, (int)sm, per};
    if (grid > 0) k<<<grid, threads, sm, st>>>(A, rhs_only);
  }
}

template <typename T>
void launch_rhs(int N, const RhsArgs<T> &A, int rhs_only, int num_sms, cudaStream_t st, LaunchInfo *info) {
  switch (N) {
    case 1: rhs_launch_n<T, 1>(A, rhs_only, num_sms, st, info); break;
    case 2: rhs_launch_n<T, 2>(A, rhs_only, num_sms, st, info); break;
    case 3: rhs_launch_n<T, 3>(A, rhs_only, num_sms, st, info); break;
    case 4: rhs_launch_n<T, 4>(A, rhs_only, num_sms, st, info); break;
    case 5: rhs_launch_n<T, 5>(A, rhs_only, num_sms, st, info); break;
    case 6: rhs_launch_n<T, 6>(A, rhs_only, num_sms, st, info); break;
    case 7: rhs_launch_n<T, 7>(A, rhs_only, num_sms, st, info); break;
    default: throw Error(DGK_ERR_UNSUPPORTED, "order N must be 1..7");
  }
}

template <typename T, int N>
static void diff_launch_n(const DiffArgs<T> &A, int num_sms, cudaStream_t st, LaunchInfo *info) {
  using O = Order<N>;
  using C = Cfg<N>;
  const int threads = C::THREADS;
  const size_t base = sizeof(T) * (size_t)(4 * C::TE * O::NPS);
  const size_t with = base + sizeof(T) * 3 * O::NP * Pad<O::NP>::V;
  if (with <= 160 * 1024) {
    auto k = diff_kernel<T, N, true>;
    const int per = std::max(1, resident(k, threads, with));
    const int grid = std::min(A.ntiles, per * num_sms);
    if (info) *info = {grid, threads, (int)with, per};
    if (grid > 0) k<<<grid, threads, with, st>>>(A);
  } else {
    auto k = diff_kernel<T, N, false>;
    const int per = std::max(1, resident(k, threads, base));
    const int grid = std::min(A.ntiles, per * num_sms);
    if (info) *info = {grid, threads, (int)base, per};
    if (grid > 0) k<<<grid, threads, base, st>>>(A);
  }
}

template <typename T>
void launch_diff(int N, const DiffArgs<T> &A, int num_sms, cudaStream_t st, LaunchInfo *info) {
  switch (N) {
    case 1: diff_launch_n<T, 1>(A, num_sms, st, info); break;
    case 2: diff_launch_n<T, 2>(A, num_sms, st, info); break;
    case 3: diff_launch_n<T, 3>(A, num_sms, st, info); break;
    case 4: diff_launch_n<T, 4>(A, num_sms, st, info); break;
    case 5: diff_launch_n<T, 5>(A, num_sms, st, info); break;
    case 6: diff_launch_n<T, 6>(A, num_sms, st, info); break;
    case 7: diff_launch_n<T, 7>(A, num_sms, st, info); break;
    default: throw Error(DGK_ERR_UNSUPPORTED, "order N must be 1..7");
  }
}

template <typename T>
void launch_update(const Tile *tiles, int ntiles, int np, T *u, T *resu, const T *rhs, double c0, double c1, double c2,
                   int mode, int num_sms, cudaStream_t st) {
  const int grid = std::min(ntiles, num_sms * 8);
  if (grid > 0) update_kernel<T><<<grid, 256, 0, st>>>(tiles, ntiles, np, u, resu, rhs, (T)c0, (T)c1, (T)c2, mode);
}

template void launch_rhs<double>(int, const RhsArgs<double> &, int, int, cudaStream_t, LaunchInfo *);
template void launch_rhs<float>(int, const RhsArgs<float> &, int, int, cudaStream_t, LaunchInfo *);
template void launch_diff<double>(int, const DiffArgs<double> &, int, cudaStream_t, LaunchInfo *);
template void launch_diff<float>(int, const DiffArgs<float> &, int, cudaStream_t, LaunchInfo *);
template void launch_update<double>(const Tile *, int, int, double *, double *, const double *, double, double, double,
                                    int, int, cudaStream_t);
template void launch_update<float>(const Tile *, int, int, float *, float *, const float *, double, double, double, int,
                                   int, cudaStream_t);

int tile_elems(int N) {
  switch (N) {
    case 1: return Cfg<1>::TE;
    case 2: return Cfg<2>::TE;
    case 3: return Cfg<3>::TE;
    case 4: return Cfg<4>::TE;
    case 5: return Cfg<5>::TE;
    case 6: return Cfg<6>::TE;
    case 7: return Cfg<7>::TE;
    default: throw Error(DGK_ERR_UNSUPPORTED, "order N must be 1..7");
  }
}

}  // namespace dgk
