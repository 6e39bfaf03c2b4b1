// FP64 setup on the GPU: node coordinates, geometric factors, normals/Fscale and the face maps of
// NewDG3D (element/library/gonudg/startup3d.go:121-148, normals3d.go:11-207, buildmaps3d.go:5-153),
// plus the generic MATMUL operator and the seeded initial fields.
#include <cstdint>

#include "kernels.hpp"
#include "runner.hpp"

namespace dgk {

// Physical coordinate of reference node j of element e (startup3d.go:126-148).
__device__ __forceinline__ void node_xyz(const GeoSetup &g, int64_t e, int j, double &x, double &y, double &z) {
  const double r = g.rst[j], s = g.rst[g.Np + j], t = g.rst[2 * g.Np + j];
  const int64_t va = g.EToV[e * 4], vb = g.EToV[e * 4 + 1], vc = g.EToV[e * 4 + 2], vd = g.EToV[e * 4 + 3];
  const double ca = -(1.0 + r + s + t), cb = 1.0 + r, cc = 1.0 + s, cd = 1.0 + t;
  x = 0.5 * (ca * g.VX[va] + cb * g.VX[vb] + cc * g.VX[vc] + cd * g.VX[vd]);
  y = 0.5 * (ca * g.VY[va] + cb * g.VY[vb] + cc * g.VY[vc] + cd * g.VY[vd]);
  z = 0.5 * (ca * g.VZ[va] + cb * g.VZ[vb] + cc * g.VZ[vc] + cd * g.VZ[vd]);
}

// J and the nine metric terms at node i of element e (normals3d.go:11-79): xr = Dr X etc.
__device__ void node_metrics(const GeoSetup &g, int64_t e, int i, double m[10]) {
  double xr = 0, xs = 0, xt = 0, yr = 0, ys = 0, yt = 0, zr = 0, zs = 0, zt = 0;
  for (int j = 0; j < g.Np; ++j) {
    double x, y, z;
    node_xyz(g, e, j, x, y, z);
    const double dr = g.Dr[i * g.Np + j], ds = g.Ds[i * g.Np + j], dt = g.Dt[i * g.Np + j];
    xr += dr * x; xs += ds * x; xt += dt * x;
    yr += dr * y; ys += ds * y; yt += dt * y;
    zr += dr * z; zs += ds * z; zt += dt * z;
  }
  const double J = xr * (ys * zt - zs * yt) - yr * (xs * zt - zs * xt) + zr * (xs * yt - ys * xt);
  m[0] = J;
  m[1] = (ys * zt - zs * yt) / J;    // rx
  m[2] = -(xs * zt - zs * xt) / J;   // ry
  m[3] = (xs * yt - ys * xt) / J;    // rz
  m[4] = -(yr * zt - zr * yt) / J;   // sx
  m[5] = (xr * zt - zr * xt) / J;    // sy
  m[6] = -(xr * yt - yr * xt) / J;   // sz
  m[7] = (yr * zs - zr * ys) / J;    // tx
  m[8] = -(xr * zs - zr * xs) / J;   // ty
  m[9] = (xr * ys - yr * xs) / J;    // tz
}

__global__ void geo_node_kernel(GeoSetup g, int which, double *out, int *status) {
  const int64_t n = g.K * g.Np;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n; idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = idx / g.Np;
    const int i = (int)(idx - e * g.Np);
    if (which < 3) {
      double x, y, z;
      node_xyz(g, e, i, x, y, z);
      out[idx] = which == 0 ? x : which == 1 ? y : z;
      continue;
    }
    double m[10];
    node_metrics(g, e, i, m);
    if (!(m[0] > 0.0)) atomicExch(status, 3);  // the reference rejects J <= 0 (normals3d.go:38-40)
    out[idx] = which == 12 ? m[0] : m[which - 2];
  }
}

// Face normals from the metric rows, normalised; sJ = |n| J and Fscale = sJ / J (normals3d.go:82-207).
__global__ void geo_face_kernel(GeoSetup g, int which, double *out) {
  const int NF = 4 * g.Nfp;
  const int64_t n = g.K * NF;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n; idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = idx / NF;
    const int q = (int)(idx - e * NF), f = q / g.Nfp;
    double m[10];
    node_metrics(g, e, g.fmask[q], m);
    double nx, ny, nz;
    if (f == 0) {
      nx = -m[7]; ny = -m[8]; nz = -m[9];
    } else if (f == 1) {
      nx = -m[4]; ny = -m[5]; nz = -m[6];
    } else if (f == 2) {
      nx = m[1] + m[4] + m[7]; ny = m[2] + m[5] + m[8]; nz = m[3] + m[6] + m[9];
    } else {
      nx = -m[1]; ny = -m[2]; nz = -m[3];
    }
    const double mag = sqrt(nx * nx + ny * ny + nz * nz);
    const double sJ = mag * m[0];
    double v;
    switch (which) {
      case 13: v = nx / mag; break;
      case 14: v = ny / mag; break;
      case 15: v = nz / mag; break;
      case 16: v = sJ; break;
      default: v = sJ / m[0];
    }
    out[idx] = v;
  }
}

__device__ __forceinline__ double wrap(double d, double L) {
  if (L > 0.0) {
    if (d > 0.5 * L) d -= L;
    if (d < -0.5 * L) d += L;
  }
  return d;
}

// VmapM / VmapP by nearest neighbour-face node within NODETOL^2 = 1e-14 (buildmaps3d.go:5-153); with a
// period, coordinate differences are wrapped into [-L/2, L/2] first.
__global__ void maps_kernel(GeoSetup g, int64_t *vmapM, int64_t *vmapP) {
  const int NF = 4 * g.Nfp;
  const int64_t n = g.K * NF;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n; idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = idx / NF;
    const int q = (int)(idx - e * NF), f = q / g.Nfp;
    const int64_t self = g.fmask[q] + e * g.Np;
    if (vmapM) vmapM[idx] = self;
    const int64_t k2 = g.EToE[e * 4 + f];
    const int f2 = (int)g.EToF[e * 4 + f];
    int64_t match = self;
    if (!(k2 == e && f2 == f) && k2 >= 0 && k2 < g.K) {
      double x1, y1, z1;
      node_xyz(g, e, g.fmask[q], x1, y1, z1);
      double best = 0.0;
      int jbest = 0;
      for (int j = 0; j < g.Nfp; ++j) {
        double x2, y2, z2;
        node_xyz(g, k2, g.fmask[f2 * g.Nfp + j], x2, y2, z2);
        const double dx = wrap(x2 - x1, g.period), dy = wrap(y2 - y1, g.period), dz = wrap(z2 - z1, g.period);
        const double d = dx * dx + dy * dy + dz * dz;
        if (j == 0 || d < best) {
          best = d;
          jbest = j;
        }
      }
      if (best < 1e-7 * 1e-7) match = g.fmask[f2 * g.Nfp + jbest] + k2 * g.Np;
    }
    vmapP[idx] = match;
  }
}

// Minimum node-pair distance of each element (examples/3d_scalar_burgers_equation.go:697-717).
__global__ void hmin_kernel(GeoSetup g, unsigned long long *dmin) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < g.K; e += (int64_t)gridDim.x * blockDim.x) {
    double best = 1e300;
    for (int i = 0; i < g.Np; ++i) {
      double xi, yi, zi;
      node_xyz(g, e, i, xi, yi, zi);
      for (int j = i + 1; j < g.Np; ++j) {
        double xj, yj, zj;
        node_xyz(g, e, j, xj, yj, zj);
        const double d = sqrt((xj - xi) * (xj - xi) + (yj - yi) * (yj - yi) + (zj - zi) * (zj - zi));
        if (d > 1e-12 && d < best) best = d;
      }
    }
    atomicMin(dmin, (unsigned long long)__double_as_longlong(best));
  }
}

static int grid_for(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 32); }

void launch_geo_field(const GeoSetup &g, int which, double *out, cudaStream_t st) {
  if (which <= 12) {
    int *status = nullptr;
    cuda_check(cudaMallocAsync(reinterpret_cast<void **>(&status), sizeof(int), st), "status");
    cuda_check(cudaMemsetAsync(status, 0, sizeof(int), st), "status");
    geo_node_kernel<<<grid_for(g.K * g.Np), 256, 0, st>>>(g, which, out, status);
    int h = 0;
    cuda_check(cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, st), "status");
    cuda_check(cudaStreamSynchronize(st), "sync");
    cudaFreeAsync(status, st);
    if (h) throw Error(DGK_ERR_INVALID, "negative Jacobian in the mesh (J <= 0)");
  } else {
    geo_face_kernel<<<grid_for(g.K * 4 * g.Nfp), 256, 0, st>>>(g, which, out);
  }
  cuda_check(cudaGetLastError(), "geometry kernel");
}

void launch_build_maps(const GeoSetup &g, int64_t *vmapM, int64_t *vmapP, cudaStream_t st) {
  maps_kernel<<<grid_for(g.K * 4 * g.Nfp), 256, 0, st>>>(g, vmapM, vmapP);
  cuda_check(cudaGetLastError(), "maps kernel");
}

void launch_hmin(const GeoSetup &g, unsigned long long *dmin, cudaStream_t st) {
  hmin_kernel<<<grid_for(g.K), 256, 0, st>>>(g, dmin);
  cuda_check(cudaGetLastError(), "hmin kernel");
}

// Generic MATMUL_<M>: one block per (element chunk, partition); M row-major in global memory (L1-cached).
template <typename T>
__global__ void matmul_kernel(const T *__restrict__ M, int rows, int cols, const T *__restrict__ in, T *out,
                              const int64_t *in_off, const int64_t *out_off, const int64_t *K, int chunk, int add) {
  const int p = blockIdx.y;
  const int64_t e0 = (int64_t)blockIdx.x * chunk, kp = K[p];
  for (int idx = threadIdx.x; idx < chunk * rows; idx += blockDim.x) {
    const int64_t e = e0 + idx / rows;
    const int i = idx % rows;
    if (e >= kp) continue;
    const T *x = in + in_off[p] + e * cols;
    T sum = T(0);
    for (int j = 0; j < cols; ++j) sum += M[i * cols + j] * x[j];
    T *o = out + out_off[p] + e * rows + i;
    *o = add ? *o + sum : sum;
  }
}

template <typename T>
void launch_matmul(const T *M, int rows, int cols, const T *in, T *out, const int64_t *d_in_off,
                   const int64_t *d_out_off, const int64_t *d_K, int npart, int64_t kmax, int add, cudaStream_t st) {
  const int chunk = std::max(1, 256 / rows);
  const int64_t gx = (kmax + chunk - 1) / chunk;
  if (gx == 0) return;
  if (gx > 0x7fffffff || npart > 65535) throw Error(DGK_ERR_UNSUPPORTED, "matmul grid too large");
  matmul_kernel<T><<<dim3((unsigned)gx, (unsigned)npart), 256, 0, st>>>(M, rows, cols, in, out, d_in_off, d_out_off,
                                                                         d_K, chunk, add);
  cuda_check(cudaGetLastError(), "matmul kernel");
}
template void launch_matmul<double>(const double *, int, int, const double *, double *, const int64_t *,
                                    const int64_t *, const int64_t *, int, int64_t, int, cudaStream_t);
template void launch_matmul<float>(const float *, int, int, const float *, float *, const int64_t *, const int64_t *,
                                   const int64_t *, int, int64_t, int, cudaStream_t);

}  // namespace dgk

namespace dgk {

// Seeded initial fields evaluated at the node coordinates:
//   kind 0: mean + amp sin(pi x) sin(pi y) sin(pi z)
//   kind 1: mean + amp sin(pi x) cos(pi y) sin(pi z)
//   kind 2: mean + sum_m a_m cos(pi (k_m . x) + phi_m), modes (kx, ky, kz, a, phi) per row
template <typename T>
__global__ void field_kernel(T *u, const T *X, const T *Y, const T *Z, int64_t n, int kind, double mean, double amp,
                             const double *modes, int nmodes) {
  const double pi = 3.141592653589793;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double x = X[i], y = Y[i], z = Z[i];
    double v = mean;
    if (kind == 0) {
      v += amp * sin(pi * x) * sin(pi * y) * sin(pi * z);
    } else if (kind == 1) {
      v += amp * sin(pi * x) * cos(pi * y) * sin(pi * z);
    } else {
      for (int m = 0; m < nmodes; ++m) {
        const double *md = modes + 5 * m;
        v += md[3] * cos(pi * (md[0] * x + md[1] * y + md[2] * z) + md[4]);
      }
    }
    u[i] = (T)v;
  }
}

template <typename T>
void launch_field(T *u, const T *X, const T *Y, const T *Z, int64_t n, int kind, double mean, double amp,
                  const double *modes, int nmodes, cudaStream_t st) {
  if (n <= 0) return;
  field_kernel<T><<<grid_for(n), 256, 0, st>>>(u, X, Y, Z, n, kind, mean, amp, modes, nmodes);
  cuda_check(cudaGetLastError(), "field kernel");
}
template void launch_field<double>(double *, const double *, const double *, const double *, int64_t, int, double,
                                   double, const double *, int, cudaStream_t);
template void launch_field<float>(float *, const float *, const float *, const float *, int64_t, int, double, double,
                                  const double *, int, cudaStream_t);

}  // namespace dgk
