/*
 * dgk.h — C ABI of the B200 (sm_100a) backend for DGKernel's partition-parallel tet-DG right-hand side.
 *
 * The entry points replace the gocca/OCCA device layer under DGKernel's Go `runner` package for the
 * named RHS kernels; every entry point cites the reference interface it stands in for (paths relative to
 * the DGKernel project root).  All calls return an int status (DGK_OK = 0); the message of the last
 * failure is available from dgk_last_error() (per runner) or dgk_global_error() (calls without a runner).
 *
 * Ownership: host pointers are used only for the duration of a call and never retained (cgo forbids C
 * from keeping Go pointers).  Device memory is owned by the runner and released by dgk_runner_free.
 * Threading: a runner is not thread-safe; all of its work is ordered on one CUDA stream.  Unlike the
 * reference's ExecuteKernel, which calls Device.Finish() after every kernel
 * (runner/kernel_execution.go:62), dgk_execute_kernel only synchronises when the configuration asks for
 * a copy back; dgk_sync() is the explicit Finish.
 */
#ifndef DGK_H
#define DGK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------------------ */
#define DGK_OK 0
#define DGK_ERR_INVALID 1     /* bad argument; also the reference's panics (empty K, KpartMax > 2^20) */
#define DGK_ERR_STATE 2       /* call out of order (define after allocate, execute before build, ...) */
#define DGK_ERR_NOT_FOUND 3   /* unknown binding / kernel / op */
#define DGK_ERR_CUDA 4        /* a CUDA runtime call failed */
#define DGK_ERR_TIMEOUT 5     /* a device-side bounded wait gave up (status word set by the kernel) */
#define DGK_ERR_UNSUPPORTED 6 /* valid request this backend does not implement */
#define DGK_ERR_NO_DEVICE 7   /* no CUDA device: the backend has no CPU fallback */

/* ---- enumerations mirroring runner/builder ------------------------------------------------------ */
/* builder.DataType (runner/builder/builder.go:12-20) */
#define DGK_FLOAT32 1
#define DGK_FLOAT64 2
#define DGK_INT32 3
#define DGK_INT64 4
/* builder.Direction (runner/builder/builder_param.go:10-17) */
#define DGK_INPUT 0
#define DGK_OUTPUT 1
#define DGK_INOUT 2
#define DGK_TEMP 3
#define DGK_SCALAR 4
/* runner.ActionFlags (runner/binding.go:15-26): CopyTo = 1<<1, CopyBack = 1<<2 */
#define DGK_NO_ACTION 0
#define DGK_COPY_TO 2
#define DGK_COPY_BACK 4
#define DGK_COPY 6
/* host layout of an array binding: flat []T (element-contiguous already), or a row-major gonum
 * mat.Matrix rows x cols that copies transpose to column-major (runner/kernel_copy.go:86-111) */
#define DGK_LAYOUT_FLAT 0
#define DGK_LAYOUT_MATRIX 1

typedef struct dgk_runner dgk_runner;
typedef struct dgk_element dgk_element;
typedef struct dgk_graph dgk_graph;

/* ---- runner lifecycle --------------------------------------------------------------------------- */
/* NewRunner + builder.NewBuilder (runner/runner.go:48-86, runner/builder/builder.go:73-100).
 * int_type is DGK_INT32 or DGK_INT64 (0 = INT64).  Fails with DGK_ERR_INVALID for npart < 1 or
 * KpartMax > 2^20 (the reference panics), DGK_ERR_NO_DEVICE without a GPU. */
int dgk_runner_create(const int64_t *K, int32_t npart, int32_t int_type, dgk_runner **out);
/* A runner that plans without a device: bindings, aligned offsets, kernel signatures and the preamble
 * work; copies, BuildKernel and ExecuteKernel fail with DGK_ERR_NO_DEVICE.  For host-side tooling. */
int dgk_runner_create_host_only(const int64_t *K, int32_t npart, int32_t int_type, dgk_runner **out);
/* Runner.Free (runner/runner.go:178-188). */
int dgk_runner_free(dgk_runner *r);
const char *dgk_last_error(const dgk_runner *r);
const char *dgk_global_error(void);
/* Use an existing cudaStream_t (as void*) for all work of this runner; NULL = the runner's own. */
int dgk_set_stream(dgk_runner *r, void *cuda_stream);
/* Device.Finish (runner/kernel_execution.go:62). */
int dgk_sync(dgk_runner *r);

/* ---- captured launch sequences ------------------------------------------------------------------- */
/* No counterpart in the reference, whose ExecuteKernel (runner/kernel_execution.go:12-89) runs one kernel
 * per call.  Record nlaunch (even, >= 2) consecutive launches of a built kernel, launch l taking the
 * nscalars values at scalars + l*nscalars, into one CUDA graph on the runner's stream; nothing runs until
 * dgk_graph_launch.  Operators that alternate ping-pong buffers swap them once per recorded launch, so
 * after every replay the bindings name the newest state.  The kernel's configuration may carry no host
 * copies.  A graph is tied to its runner: free it before the runner. */
int dgk_capture_graph(dgk_runner *r, const char *kernel_name, int32_t nlaunch, int32_t nscalars,
                      const double *scalars, dgk_graph **out);
/* Launch a captured sequence `repeats` times on the runner's stream (asynchronous; dgk_sync reports the
 * kernels' status word). */
int dgk_graph_launch(dgk_graph *g, int32_t repeats);
int dgk_graph_free(dgk_graph *g);

/* ---- bindings (DefineBindings, runner/binding.go:100-195) --------------------------------------- */
/* Array or temp binding.  part_values (part_count entries) gives the host values of each partition of a
 * [][]T / []mat.Matrix binding; part_count 0 means non-partitioned.  A partitioned runner rejects
 * non-partitioned arrays and a partition-count mismatch (binding.go:181-191).  layout/rows/cols describe
 * a mat.Matrix host binding (rows x cols per partition for []mat.Matrix).  align is the
 * builder.AlignmentType in bytes (0 or 1 = none). */
int dgk_bind_array(dgk_runner *r, const char *name, int32_t dir, int32_t host_dtype, int32_t dev_dtype,
                   int64_t total_values, int32_t part_count, const int64_t *part_values, int32_t align, int32_t layout,
                   int64_t rows, int64_t cols);
/* Input(name).Bind(mat).ToMatrix()[.Static()] (runner/binding.go:422-488).  Values row-major; stored on
 * the device column-major (runner/runner.go:375-417).  dev_dtype FLOAT64/FLOAT32, or INT32 for integer
 * tables such as Fmask. */
int dgk_bind_matrix(dgk_runner *r, const char *name, int64_t rows, int64_t cols, const double *rowmajor,
                    int32_t is_static, int32_t dev_dtype);
/* Scalar(name)[.Bind(v)] (runner/builder/builder_param.go:86-95).  bound_value NULL = unbound. */
int dgk_bind_scalar(dgk_runner *r, const char *name, int32_t dtype, const double *bound_value);
/* AllocateDevice (runner/binding.go:339-384): one pooled device arena, aligned per-partition offsets
 * (runner/builder/builder.go:113-159). */
int dgk_allocate(dgk_runner *r);

/* ---- copies (runner/memory_operations.go, runner/kernel_copy.go, runner/runner_copy.go) ----------- */
/* CopyToDevice / CopyFromDevice of a whole binding (memory_operations.go:219-241).  The host buffer holds
 * every partition back to back in the host type and layout; conversion f64<->f32 / i64<->i32 and the
 * mat.Matrix transpose run on the GPU.  bytes must equal the binding's host size. */
int dgk_copy_to_device(dgk_runner *r, const char *name, const void *host, int64_t bytes);
int dgk_copy_from_device(dgk_runner *r, const char *name, void *host, int64_t bytes);
/* One partition of a [][]T / []mat.Matrix binding (kernel_copy.go:288-560), the cgo-safe form. */
int dgk_copy_partition_to_device(dgk_runner *r, const char *name, int32_t part, const void *host, int64_t bytes);
int dgk_copy_partition_from_device(dgk_runner *r, const char *name, int32_t part, void *host, int64_t bytes);
/* Raw device bytes of an array starting at a value offset, in the device type and layout (gocca
 * Memory.CopyToWithOffset as used by CopyArrayToHost / CopyPartitionToHost, runner/runner_copy.go:13-145). */
int dgk_copy_raw_from_device(dgk_runner *r, const char *name, int64_t value_offset, void *host, int64_t bytes);
/* Host-side copy of `<name>_offsets` (runner/runner.go:227-254), npart+1 values. */
int dgk_get_offsets(dgk_runner *r, const char *name, int64_t *out);
/* Device address of `<name>_global` (or of a matrix), for zero-copy interop. */
int dgk_device_ptr(dgk_runner *r, const char *name, void **out);

/* ---- kernels (runner/kernel_config.go, runner/kernel_execution.go, runner/runner.go:88-126) ------- */
/* ConfigureKernel(name, Param(p).CopyTo()...) (kernel_config.go:51-91). */
int dgk_configure_kernel(dgk_runner *r, const char *kname, int32_t nparams, const char *const *params,
                         const uint32_t *actions);
/* BuildKernel(src, name) (runner/runner.go:88-126): selects the precompiled sm_100a operator `op_id`
 * ("differentiate", "computeRHS", "updateSolution", "rhsStage", "rhsLF", "lserkUpdate", "matmul",
 * "matmulAdd", "faceGather") instead of JIT-compiling OKL.  Operator roles bind to configured parameters
 * by name; `op_id` may carry explicit role=binding pairs, e.g. "matmul(M=Dr_NudgTet2,IN=U,OUT=Ur)". */
int dgk_build_kernel(dgk_runner *r, const char *kname, const char *op_id);
/* ExecuteKernel(name, scalars...) (kernel_execution.go:12-89): pre-copies (CopyTo), launch, post-copies
 * (CopyBack).  host_ptrs[i] is the host buffer of configured parameter i (NULL = no copy).  Scalars are
 * resolved as the reference does: a bound value first, then the positional list (kernel_execution.go:
 * 114-138). */
int dgk_execute_kernel(dgk_runner *r, const char *kname, int32_t nscalars, const double *scalars,
                       void *const *host_ptrs);
/* GetKernelSignatureForConfig (kernel_execution.go:230-237, kernel_config.go:183-246): OKL argument list. */
int dgk_kernel_signature(dgk_runner *r, const char *kname, char *buf, int64_t buflen);
/* GeneratePreamble (runner/builder/builder.go:172-410): the text the reference prepends to OKL. */
int dgk_generate_preamble(dgk_runner *r, char *buf, int64_t buflen);

/* ---- reference element (element/library/gonudg: startup3d.go, lift3d.go, nodes3d.go) -------------- */
/* NewDG3D's mesh-independent operators for order N (1..8), FP64 on the host. */
int dgk_element_create(int32_t N, dgk_element **out);
int dgk_element_free(dgk_element *e);
int dgk_element_dims(const dgk_element *e, int32_t *Np, int32_t *Nfp);
/* Row-major copy of "r","s","t" (Np), "V","Vinv","MassMatrix","M","Minv","Dr","Ds","Dt" (Np x Np) or
 * "LIFT" (Np x 4Nfp); names as GetRefMatrices (tetnudg/tet_nudg_mesh.go:371-389). */
int dgk_element_get(const dgk_element *e, const char *what, double *out, int64_t count);
/* Fmask, 4 x Nfp (startup3d.go:179-209). */
int dgk_element_fmask(const dgk_element *e, int32_t *out);

/* ---- mesh, connectivity and face maps ------------------------------------------------------------ */
/* Structured n^3 Kuhn-cube mesh on [lo,hi]^3 (6 tets per cube, utils/mesh_test_helpers.go:346-388
 * order), cubes x-slowest, EToP = x-slab of nslab slabs.  VX/VY/VZ: (n+1)^3; EToV, EToV_periodic
 * (vertex ids wrapped mod n for periodic face matching) and EToP: 6n^3 entries (EToV 4 per element). */
int dgk_kuhn_mesh(int32_t n, int32_t nslab, double lo, double hi, double *VX, double *VY, double *VZ,
                  int64_t *EToV, int64_t *EToV_periodic, int64_t *EToP);
/* Gambit neutral mesh file, tetrahedra only (replaces ReadGambitNeutral, mesh/readers/gambit_reader.go:13-338).
 * First call with NULL arrays: counts[4] = {vertices, elements, boundary faces, has_partitions}.  Second call
 * with arrays of those sizes: VX/VY/VZ (vertices in file order), EToV (4 per element, 0-based vertex
 * positions), EToP (partition N of every element in a group named "p<N>", -1 for unassigned elements; written
 * only when has_partitions, i.e. the file has more than one element group), bfaces (3 per boundary face:
 * element, 0-based Gambit face, boundary-set index).  Elements other than 4-node tetrahedra are an error. */
int dgk_read_gambit(const char *path, int64_t *counts, double *VX, double *VY, double *VZ, int64_t *EToV,
                    int64_t *EToP, int64_t *bfaces);
/* tiConnect3D (element/library/gonudg/ticonnect3d.go:24-102). */
int dgk_ti_connect3d(int64_t K, const int64_t *EToV, int64_t *EToE, int64_t *EToF);
/* FaceConnector (utils/face_connector.go:43-187).  First call with pick_idx == NULL to get the
 * (npart*npart) list lengths in pick_len (pick_len[src*npart+dst] == place_len[dst*npart+src]); then
 * call again with pick_idx/place_idx sized to the sums to receive the lists, CSR-concatenated in pair
 * order.  Verify (face_connector.go:208-253) runs on every build. */
int dgk_face_connector(int64_t K, int32_t Nfaces, int32_t Nfp, int32_t Np, const int64_t *vmapP,
                       const int64_t *EToP, int32_t npart, int64_t *pick_len, int64_t *pick_idx,
                       int64_t *place_idx);
/* Slab exchange plan of one rank (the FaceConnector pick -> exchange -> place of utils/face_connector.go:143-187
 * across ranks; partitions/gather_scatter_array_design.md:176-228).  Partition p lives on rank part_rank[p];
 * the rank's state array holds its partitions at local_off[0..L-1] and a halo at local_off[L].  First call
 * with gmap == NULL: counts[0] = face points of the rank (gmap length), counts[1] = halo values, counts[2] =
 * values sent.  Second call: gmap (int32, the rank's face points partition by partition, remote neighbours
 * pointing into the halo), send_idx (local value indices to pack, peer by peer ascending), and per peer rank
 * send_count, recv_count, recv_off (offset in the halo).  Wire order for each (sender, receiver): destination
 * partitions ascending, source partitions ascending, pick order within a pair. */
int dgk_halo_plan(int64_t K, int32_t Nfaces, int32_t Nfp, int32_t Np, const int64_t *vmapP, const int64_t *EToP,
                  int32_t npart, const int32_t *part_rank, int32_t nranks, int32_t rank, const int64_t *local_off,
                  int64_t *counts, int32_t *gmap, int64_t *send_idx, int64_t *send_count, int64_t *recv_count,
                  int64_t *recv_off);
/* Pack step of the exchange: dst[i] = src[idx[i]] for i < n, values of dtype (DGK_FLOAT32 / DGK_FLOAT64), all
 * pointers device memory, on cuda_stream.  An index outside [0, src_count) yields 0 (no read). */
int dgk_gather_values(const void *src, int32_t dtype, int64_t src_count, const int64_t *idx, int64_t n, void *dst,
                      void *cuda_stream);
/* Fused pick->exchange->place gather map: for every face point of partition p (in that partition's
 * P-buffer order), the absolute value index of its neighbour node in an array whose partition p starts
 * at node_off[p].  This is the one-address-space form of the FaceConnector exchange. */
int dgk_face_gather_map(int64_t K, int32_t Nfaces, int32_t Nfp, int32_t Np, const int64_t *vmapP,
                        const int64_t *EToP, int32_t npart, const int64_t *node_off, int32_t *gmap);
/* Compact face connectivity of the mixed stage (rhsStageMixed), derived from a gather map as above: per
 * element slot 5 int32 = the value index of each face's neighbour's first node and four packed 8-bit
 * face-order codes, partition p's elements at slots sum_{q<p} roundup32(K[q]) + e; table_out[code*Nfp + i]
 * = node index of face point i within the neighbour (table_cap codes of room).  gmap holds partition p's
 * face points at face_off[p]; node_off[p] is where partition p starts in the state array.  Every gmap entry
 * equals base + table[code][i] for its face (checked).  A derived form of the FaceConnector pick/place
 * lists (utils/face_connector.go:143-205); the reference has no compact form. */
int dgk_compact_faces(int32_t npart, const int64_t *K, const int64_t *node_off, const int64_t *face_off,
                      int32_t Np, int32_t Nfp, const int32_t *gmap, int32_t *conn_out, uint8_t *table_out,
                      int32_t table_cap, int32_t *ncodes_out);
/* Tiles of the tensor-core mixed stage (rhsStageMixed mma=1) with their halos, from the compact connectivity
 * above (conn in dgk_compact_faces' slot layout).  Each partition is cut into runs of consecutive elements of
 * at most max_elems, starting on multiples of `align`, with at most max_halo (even) faces whose neighbour lies
 * outside the run.  Call once with the output pointers NULL to get counts_out = {tiles, halo entries}, then
 * again with room for them: per tile part_out, first_out (partition-local first element), nelem_out,
 * halo_off_out (tiles + 1, in entries); halo_list_out holds (neighbour base, code) int32 pairs, each tile's
 * list padded to an even count by repeating its last entry; tconn_out (4 per element slot) = the neighbour
 * trace's position in the tile's shared-memory slot (low 16 bits, floats: (neighbour - first) * Np inside
 * the tile, halo_floats + j * Nfp for halo face j) | code << 16 (identity_code for halo faces).  Derived from
 * the FaceConnector lists (utils/face_connector.go:143-205); the reference has no tiled form. */
int dgk_tile_halo(int32_t npart, const int64_t *K, const int64_t *node_off, int32_t Np, int32_t Nfp,
                  const int32_t *conn, int32_t max_elems, int32_t max_halo, int32_t halo_floats, int32_t identity_code,
                  int32_t align, int64_t *counts_out, int32_t *part_out, int64_t *first_out, int32_t *nelem_out,
                  int32_t *halo_off_out, int32_t *halo_list_out, uint32_t *tconn_out);

/* GPU FP64 setup (element/library/gonudg/startup3d.go:121-148, normals3d.go:11-207,
 * buildmaps3d.go:5-153) into the runner's bound arrays.  names[] lists the target binding for each of
 * "X","Y","Z","Rx","Ry","Rz","Sx","Sy","Sz","Tx","Ty","Tz","J","nx","ny","nz","sJ","Fscale","vmapM",
 * "vmapP" (20 entries; NULL = skip).  Node arrays hold Np values and face arrays 4*Nfp values per
 * element; partitions are the contiguous element ranges of the runner's K.  period: 0 = no periodic
 * matching, else the box length used to wrap coordinate differences.  EToE/EToF as tiConnect3D.
 * hmin_out (may be NULL) receives the smallest node-pair distance
 * (examples/3d_scalar_burgers_equation.go:697-717).  vmapM/vmapP targets may be int32 or int64. */
int dgk_setup_geometry(dgk_runner *r, const dgk_element *e, int64_t nverts, const double *VX, const double *VY,
                       const double *VZ, const int64_t *EToV, const int64_t *EToE, const int64_t *EToF,
                       double period, const char *const *names, double *hmin_out);

/* ---- seeded synthetic inputs --------------------------------------------------------------------- */
/* Evaluate an initial field at the node coordinates bound as xname/yname/zname (same type and layout):
 * kind 0: mean + amp sin(pi x) sin(pi y) sin(pi z); kind 1: mean + amp sin(pi x) cos(pi y) sin(pi z);
 * kind 2: mean + sum_m a_m cos(pi (k_m . x) + phi_m) with modes rows (kx, ky, kz, a, phi). */
int dgk_init_field(dgk_runner *r, const char *name, const char *xname, const char *yname, const char *zname,
                   int32_t kind, double mean, double amp, int32_t nmodes, const double *modes);
/* As dgk_init_field with kind 2, but every partition (for example every independent instance of a batch)
 * takes its own nmodes modes: modes holds npart * nmodes rows, partition p's rows first at p * nmodes. */
int dgk_init_field_parts(dgk_runner *r, const char *name, const char *xname, const char *yname, const char *zname,
                         double mean, int32_t nmodes, const double *modes);
/* splitmix64 uniform stream (53-bit doubles), for reproducible inputs across host and oracle. */
int dgk_splitmix_uniform(uint64_t seed, int64_t count, double *out);

/* ---- shock-sensor network (learned sensor of the artificial-viscosity stage) ---------------------------
 * No counterpart in the reference, which has no sensor.  A 3-layer perceptron nin -> 32 -> 32 -> 1 (tanh,
 * tanh, sigmoid); parameters are `count` float32 values W1[32][nin], b1[32], W2[32][32], b2[32], w3[32], b3,
 * with nin = Np of orders 1..5.  All arrays are device pointers; work is queued on cuda_stream (NULL: the
 * default stream) and the calls return without synchronising. */
int dgk_mlp_param_count(int32_t nin, int64_t *count);
/* out[s] = network(X[s, :]) for n samples; fp16 = 1 rounds the weights to FP16 first (sums stay FP32, the
 * arithmetic of the stage's sensor), which needs `half_scratch` of count 2-byte values. */
int dgk_mlp_forward(const float *params, const float *X, int64_t n, int32_t nin, int32_t fp16, float *out,
                    void *half_scratch, void *cuda_stream);
/* grad = d/dparams of mean_s (network(X[s]) - y[s])^2 and loss = that mean (both overwritten). */
int dgk_mlp_loss_grad(const float *params, const float *X, const float *y, int64_t n, int32_t nin, float *grad,
                      float *loss, void *cuda_stream);
/* One Adam step (bias-corrected, step counted from 1) on `count` parameters with moments m and v. */
int dgk_mlp_adam(float *params, const float *grad, float *m, float *v, int64_t count, float lr, float beta1,
                 float beta2, float eps, int32_t step, void *cuda_stream);

/* ---- allocation-free upload ----------------------------------------------------------------------- */
/* No counterpart in the reference.  Converting upload that allocates nothing: `count` host values of
 * host_dtype are staged in a fixed 8 MiB array inside the library's device image and converted on the GPU
 * into `device_dst` (dev_dtype), on `cuda_stream` (NULL = legacy default stream); the call returns after the
 * stream has finished.  For callers that must not allocate device memory once running -- a host application
 * that owns the device-memory budget, or a time-stepping loop that cannot absorb a cudaMalloc's latency and
 * implicit synchronisation -- unlike dgk_copy_to_device, whose staging buffer grows with cudaMalloc.  More than 8 MiB of host data is rejected
 * with DGK_ERR_INVALID (split the upload).  The first call on each device resolves the array's device
 * address, so make it before any stream capture; the address is kept for the life of the process, so after a
 * cudaDeviceReset (which ends the context that holds the array) the entry point must not be called again.
 * All calls share the array: calls that overlap on the GPU race.  Errors are reported through
 * dgk_global_error(). */
int dgk_convert_upload_noalloc(const void *host, int32_t host_dtype, void *device_dst, int32_t dev_dtype,
                               int64_t count, void *cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* DGK_H */
