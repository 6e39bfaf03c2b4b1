// sm_100a kernels of the tet-DG right-hand side (plain FP64 / FP32 forms).
//
// Data layout (HBM): every node array is element-contiguous, node n of element k at k*Np + n, and every
// face array holds 4*Nfp face points per element in face-major order (the reference layout of
// element/physical_element.go:29-46).  Work is cut into tiles of up to TE consecutive elements of one
// partition; a tile's slice of each array is one contiguous run, so it is read with coalesced vector
// loads.  A persistent grid of CTAs walks the tile list; each CTA stages the reference matrices
// (Dr, Ds, Dt, LIFT) in shared memory once and reads them with warp-uniform broadcasts.
//
// Thread mapping for the element-local matrix products: thread t owns element e = t % TE of the tile and
// row group g = t / TE (RG consecutive rows), so the 32 lanes of a warp hold 32 elements and share every
// matrix entry they read.  Element-major tiles in shared memory use an odd row stride, which keeps the
// strided per-element reads of a warp free of bank conflicts.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dgk {

struct Tile {
  int64_t node_base;  // value index of the tile's first element in node arrays (Np values per element)
  int64_t face_base;  // value index of the tile's first element in face arrays (4*Nfp values per element)
  int32_t nelem;      // elements in this tile (<= TE)
  int32_t part;       // partition (or instance) the tile belongs to
};

// Status word codes written by kernels (never a trap: the host reads the word and reports).
enum : int { kStatusOk = 0, kStatusBadGather = 1 };

// Even row stride of matrices as the kernels read them (pairs of entries load as one vector).
__host__ __device__ constexpr int pad_even(int c) { return (c + 1) & ~1; }

template <int N>
struct Order {
  static constexpr int NP = (N + 1) * (N + 2) * (N + 3) / 6;
  static constexpr int NFP = (N + 1) * (N + 2) / 2;
  static constexpr int NF = 4 * NFP;
  static constexpr int NPS = NP | 1;  // odd shared-memory strides
  static constexpr int NFS = NF | 1;
};

// Launch shape per order: TE elements per tile, RG rows per thread in the matrix products.
template <int N>
struct Shape;
template <> struct Shape<1> { static constexpr int TE = 128, RG = 2; };
template <> struct Shape<2> { static constexpr int TE = 64, RG = 5; };
template <> struct Shape<3> { static constexpr int TE = 64, RG = 5; };
template <> struct Shape<4> { static constexpr int TE = 32, RG = 5; };
template <> struct Shape<5> { static constexpr int TE = 32, RG = 7; };
template <> struct Shape<6> { static constexpr int TE = 32, RG = 7; };
template <> struct Shape<7> { static constexpr int TE = 32, RG = 8; };

template <int N>
struct Cfg {
  using O = Order<N>;
  static constexpr int TE = Shape<N>::TE, RG = Shape<N>::RG;
  static constexpr int G = (O::NP + RG - 1) / RG;
  static constexpr int THREADS = TE * G;
};

// Arguments of the fused stage / RHS kernels.  Matrices are row-major in the kernel's type.
template <typename T>
struct RhsArgs {
  const Tile *tiles;
  int ntiles;
  const T *u_in;  // state read by this stage (also the neighbour traces)
  T *u_out;       // state written by this stage (ping-pong partner of u_in)
  T *resu;        // LSERK residual, updated in place
  T *rhs_out;     // RHS-only mode: the right-hand side
  const T *geo[9];       // rx, ry, rz, sx, sy, sz, tx, ty, tz per node
  const T *face[4];      // nx, ny, nz, Fscale per face point
  const int32_t *gmap;   // neighbour value index per face point (fused FaceConnector exchange)
  int64_t n_u_values;    // bound of gmap entries
  const T *Dmat;         // [3][NP][pad(NP)] Dr, Ds, Dt; rows padded to an even length (16-byte pairs)
  const T *LIFT;         // [NP][pad(NF)]
  const int32_t *fmask;  // [NF]
  T a, b, dt;            // LSERK stage coefficients
  int conservative;      // 0: -u (ux+uy+uz) (reference form), 1: -div(u^2/2 (1,1,1))
  int *status;
  // compact FP64 form (straight-sided elements): kCompactGeo64 values per element slot, compact connectivity
  // (kMixedConnWords per slot) with its face-order table, and each tile's first element slot
  const double *geoc;
  const int32_t *conn;
  const uint8_t *ftab;
  int ncodes;
  const int64_t *tile_slot;
};

// compact FP64 geometry per element: rx .. tz, then per face nx, ny, nz, Fscale
constexpr int kCompactGeo64 = 25;

template <typename T>
struct DiffArgs {
  const Tile *tiles;
  int ntiles;
  const T *u;
  const T *geo[9];
  T *out[3];   // differentiate: DuDx, DuDy, DuDz;  computeRHS: out[0] = rhsu
  int mode;    // 0 = differentiate, 1 = reference volume-only computeRHS
  const T *Dmat;  // [3][NP][pad(NP)], rows padded to an even length
};

// ---- mixed-precision stage (mixed.cu) ----
constexpr int kMixedSlotElems = 32;  // elements per ring slot (one per lane of a consumer warp)
constexpr int kMixedGeoWords = 8;    // cr, cs, ct, g_0..g_3, pad
constexpr int kMixedConnWords = 5;   // neighbour base per face, 4 packed 8-bit face-order codes

struct MTile {
  int64_t node_base;  // value index of the slot's first node in the hi/lo/resu arrays
  int64_t elem_slot;  // index of the slot's first element in the compact geometry/connectivity arrays
  int32_t nelem;      // elements in the slot (<= kMixedSlotElems)
  int32_t part;       // partition (or instance)
};

struct MixedArgs {
  const MTile *tiles;
  int ntiles;
  const float *uhi_in, *ulo_in;  // state read by this stage (hi also supplies the neighbour traces)
  float *uhi_out, *ulo_out;      // state written by this stage (ping-pong partners)
  float *resu;                   // LSERK residual, updated in place
  const float *geo;              // kMixedGeoWords per element slot
  const int32_t *conn;           // kMixedConnWords per element slot (tensor-core form: 4 tile-local words)
  int64_t n_u_values;            // bound of every gathered value index
  const float *Dm;               // [NP][NPJ][3]: Dr, Ds, Dt entries interleaved per column, zero-padded
  const float *lift;             // [NP][4 Nfp]
  const unsigned char *bmat;     // tensor-core form: split BF16 operands of D and LIFT (tcm_pack_operands)
  const int32_t *halo_off;       // tensor-core form: per tile, first entry of its halo list (ntiles + 1)
  const int32_t *halo_list;      // tensor-core form: (neighbour base, face-order code) per halo face
  const int32_t *vslot;          // tensor-core form with viscosity: per element slot, row of visc or -1
  const double *visc;            // [row][Np] viscous right-hand side added before the update
  const double *bary;            // [NP][3] barycentric weights of vertices B, C, D at each node
  const int32_t *vtx;            // node index of vertices A, B, C, D
  const uint8_t *ftab;           // [ncodes][Nfp] neighbour-local node index of each face point
  const int32_t *fmask;          // [4 Nfp]
  int ncodes, ns;                // face-order codes in use; ring slots (set by the launcher)
  float a, dt;                   // LSERK coefficients
  double b;
  int conservative;
  int *status;
};

template <typename T>
struct CompactGeoArgs {
  int npart, np, nf;
  int64_t elem_total;
  const int64_t *elem_prefix;  // device, npart+1: first global element of each partition
  const int64_t *slot_prefix;  // device, npart: first element slot of each partition (slot-padded)
  const int64_t *node_off;     // device, npart: value offset of each partition in the metric arrays
  const int64_t *face_off;     // device, npart: value offset of each partition in the face arrays
  const T *geo[9];             // rx, ry, rz, sx, sy, sz, tx, ty, tz
  const T *face[4];            // nx, ny, nz, Fscale
  float *out;                  // kMixedGeoWords per slot
  int *bad;                    // count of elements that are not affine within 1e-9
};

struct SplitJoinArgs {
  int npart, join;  // join = 0: u -> (hi, lo);  join = 1: (hi, lo) -> u
  const int64_t *count, *u_off, *hi_off, *lo_off;  // device, npart each (values)
  double *u;
  float *hi, *lo;
};

// ---- precision form with exact integer products on the tensor cores (oz.cu) ----
struct OzArgs {
  const MTile *tiles;  // tiles of up to 32 elements (one compact-geometry slot each)
  int ntiles;
  const float *uhi_in, *ulo_in;
  float *uhi_out, *ulo_out, *resu;
  const float *geo;             // kMixedGeoWords per element slot
  const int32_t *conn;          // kMixedConnWords per element slot
  int64_t n_u_values;           // bound of every gathered value index
  const unsigned char *amat;    // matrix digits in 4 KB chunks, digit-major (oz_pack_operands)
  const int32_t *rexp;          // [2][128]: row exponents of the volume and LIFT rows
  const double *bary;           // [NP][3]
  const int32_t *vtx;           // vertex nodes A..D
  const uint8_t *ftab;          // [ncodes][Nfp]
  const int32_t *fmask;         // [4 Nfp]
  int ncodes;
  double a, b, dt;
  int *status;
};

// ---- learned-sensor viscosity on the mixed stage (lsens.cu) ----
struct LsArgs {
  const MTile *tiles;  // the mixed stage's tiles (element slots)
  int ntiles;
  int npart;
  const int64_t *slot_prefix;  // device, npart + 1: first element slot of each partition
  const int64_t *kpart;        // device, npart: elements per partition
  const int64_t *uoff;         // device, npart: value offset of each partition in the state arrays
  const int64_t *goff;         // device, npart: value offset in the FP64 metric arrays
  const int64_t *foff;         // device, npart: value offset in the face arrays and the gather map
  const float *uhi, *ulo;      // the state this stage reads
  const double *geo[9];        // rx .. tz per node (FP64)
  const double *face[4];       // nx, ny, nz, Fscale per face point (FP64)
  const int32_t *gmap;         // absolute neighbour value index per face point
  const int32_t *conn;         // compact connectivity per element slot (neighbour base per face)
  int64_t n_u_values;
  const double *Dr, *Ds, *Dt, *LIFT;  // transposed: [j][i] (LIFT [m][i])
  const double *Vinv;                  // row-major [i][j]
  const int32_t *fmask, *top;
  const double *h_over_n;      // per element slot
  int mode;                    // 1 PP, 2 MLP with PP fallback, 3 as 2 with outputs <= lo read as smooth
  double eps0, s0, kappa;
  float conf_lo, conf_hi;
  const unsigned short *mlp16;
  double *eps;                 // per element slot
  int32_t *aslot;              // per element slot: index in the active list or -1
  int32_t *alist, *tflag, *vslot, *tlist;
  int32_t *counts;             // [0] active, [1] touched, [2] network fallbacks to PP
  double *eq;                  // [active][Np][3]: eps q (a node's three components adjacent)
  double *visc;                // [touched][Np]: the viscous right-hand side
  int64_t nslots;
  int *status;
};

// ---- artificial-viscosity stage and shock-sensor MLP (av.cu) ----
struct AvTile {
  int64_t node_base;  // value index of the tile's first element in node arrays
  int64_t face_base;  // value index of the tile's first element in face arrays
  int64_t elem_base;  // global index of the tile's first element (the operator's own per-element arrays)
  int64_t e1_base;    // value index in bound per-element arrays (one value per element)
  int64_t feat_base;  // value index in a bound feature array (Np values per element)
  int32_t nelem, part;
};

struct AvArgs {
  const AvTile *tiles;
  int ntiles;
  const double *u;      // state read by this stage (and the neighbour traces)
  double *u_out;        // state written (ping-pong partner)
  double *resu;         // LSERK residual, in place
  double *q[3];         // BR1 gradient (x, y, z), node arrays
  double *eps;          // viscosity per node (constant per element)
  const double *geo[9];
  const double *face[4];
  const int32_t *gmap;
  int64_t n_u_values;
  const double *Dr, *Ds, *Dt, *Vinv;  // row-major Np x Np
  const double *LIFT;                 // row-major Np x 4Nfp
  const int32_t *fmask;               // [4 Nfp]
  const int32_t *top;                 // [Np] 1 for the modes of total degree N
  const double *h_over_n;             // per element: (2 / max Fscale) / N
  int mode;                           // 0: no viscosity, 1: PP sensor, 2: MLP sensor with PP fallback
  double eps0, s0, kappa;
  float conf_lo, conf_hi;             // MLP outputs inside (lo, hi) fall back to the PP activation
  const unsigned short *mlp16;        // MLP parameters as FP16 bits
  float *S_out, *sig_out, *feat_out, *mlp_out;  // optional per-element sensor outputs
  unsigned int *fallback_count;       // optional
  double a, b, dt;
  int prep_only;                      // 1: sensor / gradient pass only
  int *status;
};

}  // namespace dgk
