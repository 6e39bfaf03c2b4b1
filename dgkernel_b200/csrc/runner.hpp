// Runner core: bindings, pooled device memory with aligned per-partition offsets, copy engine and named
// operator execution — the B200 replacement of DGKernel's runner over gocca
// (runner/runner.go, runner/binding.go, runner/kernel_config.go, runner/kernel_execution.go,
// runner/memory_operations.go, runner/kernel_copy.go).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "dgk.h"

namespace dgk {

// An error carrying a DGK status code.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

void cuda_check(cudaError_t e, const char *what);
// Message returned by dgk_global_error() for calls made without a runner.
void set_global_error(const std::string &msg);

// Values of the device status word (kernels write them, the host reads them; nothing traps).
constexpr int kStatusGatherCode = 1;   // a face gather index was out of range
constexpr int kStatusTimeoutCode = 2;  // a bounded device-side wait gave up
int dtype_size(int dtype);

struct Binding {
  std::string name;
  int dir = DGK_INPUT;
  int host_dtype = DGK_FLOAT64, dev_dtype = DGK_FLOAT64;
  int64_t total_values = 0;              // host values (all partitions)
  std::vector<int64_t> part_values;      // host values per partition (partitioned bindings)
  bool partitioned = false, is_matrix = false, is_static = false, is_scalar = false, is_temp = false;
  int layout = DGK_LAYOUT_FLAT;
  int64_t rows = 0, cols = 0;            // matrix shape (per partition for []mat.Matrix)
  int align = 1;
  bool scalar_bound = false;
  double scalar_value = 0.0;
  std::vector<double> mat;               // host copy of a bound matrix, row-major
  // device side
  char *dptr = nullptr;                  // inside the runner's arena
  size_t dbytes = 0;
  std::vector<int64_t> offsets;          // values, npart + 1 (arrays and temps)
  void *doffsets = nullptr;              // device `<name>_offsets` (int_t)
  int64_t values_per_elem = 0;           // device values per element (arrays and temps)
};

struct ParamUse {
  Binding *b;
  uint32_t actions;
};

class Runner;

// A built operator: resolves roles against a kernel configuration and launches on the runner's stream.
struct Op {
  virtual ~Op() = default;
  virtual void launch(Runner &r, const std::vector<double> &scalars) = 0;
  // Work that must happen before a stream capture records launches (function attributes and the like).
  virtual void prepare(Runner &) {}
  // Scalar names the operator consumes, in the order it expects them.
  virtual std::vector<std::string> scalar_names() const { return {}; }
};

struct KernelConfig {
  std::string name;
  std::vector<ParamUse> params;
  std::unique_ptr<Op> op;
};

class Runner {
 public:
  Runner(const int64_t *K, int npart, int int_type, bool host_only = false);
  ~Runner();

  // DefineBindings
  void bind_array(const char *name, int dir, int host_dtype, int dev_dtype, int64_t total, int part_count,
                  const int64_t *part_values, int align, int layout, int64_t rows, int64_t cols);
  void bind_matrix(const char *name, int64_t rows, int64_t cols, const double *rowmajor, int is_static, int dev_dtype);
  void bind_scalar(const char *name, int dtype, const double *bound);
  void allocate();

  // copies
  void copy_to_device(const char *name, const void *host, int64_t bytes);
  void copy_from_device(const char *name, void *host, int64_t bytes);
  void copy_partition_to_device(const char *name, int part, const void *host, int64_t bytes);
  void copy_partition_from_device(const char *name, int part, void *host, int64_t bytes);
  // Store a packed device array (element-contiguous, all partitions back to back, type src_dtype) into a
  // binding's partitioned layout, converting type on the GPU.
  void store_packed(Binding &b, const void *dsrc, int src_dtype);

  // kernels
  void configure_kernel(const char *kname, int n, const char *const *params, const uint32_t *actions);
  void build_kernel(const char *kname, const char *op_id);
  void execute_kernel(const char *kname, int nscalars, const double *scalars, void *const *host_ptrs);
  std::string kernel_signature(const char *kname);
  std::string preamble();

  Binding &binding(const std::string &name);
  Binding *find(const std::string &name);
  KernelConfig &config(const std::string &name);
  void sync();
  // A captured sequence of launches of one built kernel (stream capture -> CUDA graph), replayed as a unit.
  struct Graph {
    Runner *runner = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int nlaunch = 0;
    ~Graph();
  };
  Graph *capture_graph(const char *kname, int nlaunch, int nscalars, const double *scalars);
  void launch_graph(Graph &g, int repeats);
  void set_stream(cudaStream_t s) { stream_ = s ? s : own_stream_; }
  cudaStream_t stream() const { return stream_; }
  int *status_word() { return dstatus_; }
  void check_status(const char *what);
  // Per-launch scratch (grows, owned by the runner).
  void *scratch(size_t bytes);

  std::vector<int64_t> K;
  int npart;
  int64_t kpart_max = 0, ktotal = 0;
  int int_type;
  bool allocated = false;
  bool host_only = false;  // plans bindings/offsets/signatures; no device memory, copies or launches
  void need_device(const char *what) const;
  int num_sms = 0;
  std::string last_error;

 private:
  void host_to_partition(Binding &b, int part, const char *host, int64_t host_values);
  void partition_to_host(Binding &b, int part, char *host, int64_t host_values);
  void validate_offsets(const char *context);

  std::map<std::string, std::unique_ptr<Binding>> bindings_;
  std::vector<std::string> order_;  // definition order
  std::map<std::string, KernelConfig> configs_;
  char *arena_ = nullptr;
  void *dK_ = nullptr;
  int *dstatus_ = nullptr;
  void *scratch_ = nullptr;
  size_t scratch_bytes_ = 0;
  cudaStream_t own_stream_ = nullptr, stream_ = nullptr;
  bool validate_ = false;
};

// Operator factory (ops.cu).
std::unique_ptr<Op> make_op(Runner &r, KernelConfig &cfg, const std::string &op_id);

// Type conversion / transpose launchers (kernels.cu).
void launch_convert(const void *src, int sdt, void *dst, int ddt, int64_t n, cudaStream_t s);
void launch_transpose_convert(const void *src, int sdt, void *dst, int ddt, int64_t rows, int64_t cols, bool to_cm,
                              cudaStream_t s);

}  // namespace dgk
