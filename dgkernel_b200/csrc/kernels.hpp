// Host-side declarations of the kernel launchers (kernels.cu, setup.cu).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "dg_kernels.cuh"

namespace dgk {

struct LaunchInfo {
  int grid = 0, threads = 0, smem = 0, per_sm = 0;
};

template <typename T>
void launch_rhs(int N, const RhsArgs<T> &A, int rhs_only, int num_sms, cudaStream_t st, LaunchInfo *info);
template <typename T>
void launch_diff(int N, const DiffArgs<T> &A, int num_sms, cudaStream_t st, LaunchInfo *info);
template <typename T>
void launch_update(const Tile *tiles, int ntiles, int np, T *u, T *resu, const T *rhs, double c0, double c1, double c2,
                   int mode, int num_sms, cudaStream_t st);
int tile_elems(int N);
// TMA-pipelined form of the fused stage (kernels_tma.cu); returns false when the order has no TMA form.
template <typename T>
bool launch_rhs_tma(int N, const RhsArgs<T> &A, int rhs_only, int num_sms, cudaStream_t st, LaunchInfo *info);
template <typename T>
int tma_tile_elems(int N);  // 0 when the order has no TMA form
// FP64 form with TMA streaming and the element-local products on the FP64 tensor path (kernels_tma.cu).
bool launch_rhs_dmma(int N, const RhsArgs<double> &A, int rhs_only, int num_sms, cudaStream_t st, LaunchInfo *info);
int dmma_tile_elems(int N);  // 0 when the order has no such form

// Mixed-precision stage (mixed.cu) with 4, 8 or 11 consumer warps per CTA and at most ring_max ring slots
// (0: as many as shared memory holds); returns false when the order or the warp count has no such form.
bool launch_rhs_mixed(int N, const MixedArgs &A, int consumer_warps, int ring_max, int num_sms, cudaStream_t st,
                      LaunchInfo *info);
void prepare_rhs_mixed(int N, int consumer_warps);  // attributes, before any stream capture
uint32_t mixed_slot_bytes(int N);  // 0 when the order has no such form
// Mixed stage with the element-local products on the tensor cores (tcm.cu), orders 1..4: tiles of at most
// tcm_tile_elems() elements and tcm_halo_capacity() halo faces (tile_halo, with halo positions from
// tcm_halo_floats(N)); the operand buffer comes from tcm_pack_operands (Dr, Ds, Dt, LIFT row-major FP64).
bool tcm_supported(int N);
int tcm_tile_elems();
int tcm_halo_capacity();
int tcm_halo_floats(int N);
void tcm_pack_operands(int N, const double *Dr, const double *Ds, const double *Dt, const double *LIFT,
                       std::vector<uint16_t> &out);
// consumer_warps 8 or 16 (2 or 4 threads per element)
void prepare_rhs_tcm(int N, int consumer_warps);  // attributes, before any stream capture
bool launch_rhs_tcm(int N, const MixedArgs &A, int consumer_warps, int num_sms, cudaStream_t st, LaunchInfo *info);
template <typename T>
void launch_compact_geometry(const CompactGeoArgs<T> &g, cudaStream_t st);
// Compact FP64 geometry (kCompactGeo64 values per element slot) for the compact form of the FP64 stage;
// g.out is unused, g.bad counts elements that are not straight-sided.
void launch_compact_geo64(const CompactGeoArgs<double> &g, double *out, cudaStream_t st);
void launch_split_join(const SplitJoinArgs &a, cudaStream_t st);

// Precision form with exact integer products on the tensor cores (oz.cu): orders 4..7, tiles of
// oz_tile_elems() elements; oz_pack_operands lays out the matrix digits and the row exponents (Dr, Ds, Dt,
// LIFT row-major FP64).
bool oz_supported(int N);
int oz_tile_elems();
int oz_digits();
void oz_pack_operands(int N, const double *Dr, const double *Ds, const double *Dt, const double *LIFT,
                      std::vector<uint8_t> &digits, std::vector<int32_t> &rexp);
void prepare_rhs_oz(int N);  // attributes, before any stream capture
bool launch_rhs_oz(int N, const OzArgs &A, int conservative, int num_sms, cudaStream_t st, LaunchInfo *info);

// Learned-sensor viscosity on the tensor-core mixed stage (lsens.cu), orders 1..4.
bool ls_supported(int N);
void prepare_ls(int N);  // attributes, before any stream capture
void launch_ls(int N, const LsArgs &A, int num_sms, cudaStream_t st);

// Artificial-viscosity stage and the sensor MLP (av.cu).
void launch_av(int N, const AvArgs &A, int num_sms, cudaStream_t st);
int mlp_param_count(int nin);
int av_tile_elems(int N);  // elements per tile of the viscosity kernels
void launch_to_half(const float *in, void *out, int64_t n, cudaStream_t st);
void launch_mlp_forward(const float *p, const float *X, int64_t n, int nin, float *out, int fp16, void *half_buf,
                        cudaStream_t st);
void launch_mlp_grad(const float *p, const float *X, const float *y, int64_t n, int nin, float *grad, float *loss,
                     cudaStream_t st);
void launch_adam(float *p, const float *g, float *m, float *v, int64_t P, float lr, float b1, float b2, float eps,
                 int step, cudaStream_t st);

// Generic MATMUL_<M> over partitions: out[e*rows + i] (+)= sum_j M[i][j] in[e*cols + j].
template <typename T>
void launch_matmul(const T *M_rowmajor, int rows, int cols, const T *in, T *out, const int64_t *d_in_off,
                   const int64_t *d_out_off, const int64_t *d_K, int npart, int64_t kmax, int add, cudaStream_t st);

// FP64 geometry setup (setup.cu).  Packed element-contiguous outputs (K*Np or K*4Nfp values).
struct GeoSetup {
  int N, Np, Nfp;
  int64_t K;
  const double *VX, *VY, *VZ;  // device
  const int64_t *EToV;         // device, K*4
  const int64_t *EToE, *EToF;  // device, K*4
  const double *rst;           // device, 3*Np (r, s, t)
  const double *Dr, *Ds, *Dt;  // device, Np*Np row-major
  const int *fmask;            // device, 4*Nfp
  double period;
};
// which: 0..2 = X,Y,Z; 3..11 = rx,ry,rz,sx,sy,sz,tx,ty,tz; 12 = J (node arrays);
//        13..17 = nx, ny, nz, sJ, Fscale (face arrays)
void launch_geo_field(const GeoSetup &g, int which, double *out, cudaStream_t st);
// vmapM (global node id of each face point) and vmapP (matched neighbour node) as int64.
void launch_build_maps(const GeoSetup &g, int64_t *vmapM, int64_t *vmapP, cudaStream_t st);
// Smallest node-pair distance above 1e-12 (as an ordered 64-bit pattern of a positive double).
void launch_hmin(const GeoSetup &g, unsigned long long *dmin, cudaStream_t st);
template <typename T>
void launch_field(T *u, const T *X, const T *Y, const T *Z, int64_t n, int kind, double mean, double amp,
                  const double *modes, int nmodes, cudaStream_t st);

}  // namespace dgk
