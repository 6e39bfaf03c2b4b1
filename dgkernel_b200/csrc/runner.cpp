// Runner core (see runner.hpp).  Semantics follow DGKernel's runner package; the device layer is CUDA on
// one stream instead of gocca/OCCA.
#include "runner.hpp"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <sstream>

namespace dgk {

void cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw Error(DGK_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int dtype_size(int dt) {
  switch (dt) {
    case DGK_FLOAT32:
    case DGK_INT32:
      return 4;
    case DGK_FLOAT64:
    case DGK_INT64:
      return 8;
    default:
      throw Error(DGK_ERR_INVALID, "unknown data type " + std::to_string(dt));
  }
}

static const char *ctype(int dt) {  // runner.dataTypeToCType / TypeName (runner/types.go:24-49)
  switch (dt) {
    case DGK_FLOAT32: return "float";
    case DGK_INT32: return "int";
    case DGK_INT64: return "long";
    default: return "double";
  }
}

void Runner::need_device(const char *what) const {
  if (host_only) throw Error(DGK_ERR_NO_DEVICE, std::string(what) + " needs a device: this runner is host-only");
}

Runner::Runner(const int64_t *Kin, int np, int itype, bool ho)
    : npart(np), int_type(itype ? itype : DGK_INT64), host_only(ho) {
  if (np < 1 || Kin == nullptr) throw Error(DGK_ERR_INVALID, "K array cannot be empty");
  if (int_type != DGK_INT32 && int_type != DGK_INT64) throw Error(DGK_ERR_INVALID, "IntType must be INT32 or INT64");
  K.assign(Kin, Kin + np);
  for (int64_t k : K) {
    if (k < 0) throw Error(DGK_ERR_INVALID, "negative K value");
    kpart_max = std::max(kpart_max, k);
    ktotal += k;
  }
  if (kpart_max > (1 << 20))
    throw Error(DGK_ERR_INVALID, "KpartMax exceeds 2^20 (1048576), usually caused by unbalanced workloads. Found "
                                 "KpartMax=" + std::to_string(kpart_max) + ". Reduce partition sizes.");
  if (host_only) return;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    throw Error(DGK_ERR_NO_DEVICE, "no CUDA device available (this backend has no CPU fallback)");
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  cuda_check(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
  cuda_check(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  stream_ = own_stream_;
  // K on the device as int_t (runner/runner.go:77-84)
  const int is = int_type == DGK_INT32 ? 4 : 8;
  cuda_check(cudaMalloc(&dK_, (size_t)np * is + sizeof(int) * 4), "cudaMalloc(K)");
  std::vector<char> hk((size_t)np * is);
  for (int p = 0; p < np; ++p) {
    if (is == 4) {
      int32_t v = (int32_t)K[p];
      std::memcpy(&hk[(size_t)p * 4], &v, 4);
    } else {
      std::memcpy(&hk[(size_t)p * 8], &K[p], 8);
    }
  }
  cuda_check(cudaMemcpy(dK_, hk.data(), hk.size(), cudaMemcpyHostToDevice), "copy K");
  dstatus_ = reinterpret_cast<int *>(static_cast<char *>(dK_) + (size_t)np * is);
  cuda_check(cudaMemset(dstatus_, 0, sizeof(int) * 4), "status");
  const char *v = std::getenv("DGK_VALIDATE_OFFSETS");
  validate_ = v && v[0] == '1';
}

Runner::~Runner() {
  configs_.clear();  // operators free their own buffers first
  if (arena_) cudaFree(arena_);
  if (scratch_) cudaFree(scratch_);
  if (dK_) cudaFree(dK_);
  if (own_stream_) cudaStreamDestroy(own_stream_);
}

Binding *Runner::find(const std::string &name) {
  auto it = bindings_.find(name);
  return it == bindings_.end() ? nullptr : it->second.get();
}

Binding &Runner::binding(const std::string &name) {
  Binding *b = find(name);
  if (!b) throw Error(DGK_ERR_NOT_FOUND, "binding " + name + " not found");
  return *b;
}

static void check_new(Runner &r, std::map<std::string, std::unique_ptr<Binding>> &m, std::vector<std::string> &order,
                      const char *name) {
  if (r.allocated) throw Error(DGK_ERR_STATE, "bindings cannot be defined after AllocateDevice has been called");
  if (!name || !*name) throw Error(DGK_ERR_INVALID, "binding name is empty");
  if (m.count(name)) {  // a redefinition replaces the earlier binding (Go map assignment, binding.go:121)
    m.erase(name);
    order.erase(std::find(order.begin(), order.end(), std::string(name)));
  }
}

void Runner::bind_array(const char *name, int dir, int hdt, int ddt, int64_t total, int part_count,
                        const int64_t *part_values, int align, int layout, int64_t rows, int64_t cols) {
  check_new(*this, bindings_, order_, name);
  if (dir != DGK_INPUT && dir != DGK_OUTPUT && dir != DGK_INOUT && dir != DGK_TEMP)
    throw Error(DGK_ERR_INVALID, "invalid direction for array " + std::string(name));
  auto b = std::make_unique<Binding>();
  b->name = name;
  b->dir = dir;
  b->host_dtype = hdt ? hdt : ddt;
  b->dev_dtype = ddt ? ddt : b->host_dtype;
  dtype_size(b->host_dtype);
  dtype_size(b->dev_dtype);
  b->is_temp = dir == DGK_TEMP;
  b->layout = layout;
  b->rows = rows;
  b->cols = cols;
  b->align = align > 0 ? align : 1;
  if (part_count > 0) {
    // binding.go:181-191
    if (npart <= 1)
      throw Error(DGK_ERR_INVALID, "partitioned data " + b->name + " provided to non-partitioned kernel");
    if (part_count != npart)
      throw Error(DGK_ERR_INVALID, "partition count mismatch for " + b->name + ": expected " + std::to_string(npart) +
                                       ", got " + std::to_string(part_count));
    b->partitioned = true;
    b->part_values.assign(part_values, part_values + part_count);
    total = 0;
    for (int64_t v : b->part_values) total += v;
  } else if (npart > 1 && !b->is_temp) {
    throw Error(DGK_ERR_INVALID, "non-partitioned array " + b->name + " provided to partitioned kernel");
  }
  if (total < 0) throw Error(DGK_ERR_INVALID, "negative size for " + b->name);
  if (layout == DGK_LAYOUT_MATRIX && rows <= 0) throw Error(DGK_ERR_INVALID, "matrix layout needs rows > 0");
  b->total_values = total;
  order_.push_back(b->name);
  bindings_[b->name] = std::move(b);
}

void Runner::bind_matrix(const char *name, int64_t rows, int64_t cols, const double *rm, int is_static, int ddt) {
  check_new(*this, bindings_, order_, name);
  if (rows <= 0 || cols <= 0 || !rm) throw Error(DGK_ERR_INVALID, "invalid matrix " + std::string(name));
  auto b = std::make_unique<Binding>();
  b->name = name;
  b->dir = DGK_INPUT;
  b->is_matrix = true;
  b->is_static = is_static != 0;
  b->host_dtype = DGK_FLOAT64;
  b->dev_dtype = ddt ? ddt : DGK_FLOAT64;
  dtype_size(b->dev_dtype);
  b->rows = rows;
  b->cols = cols;
  b->total_values = rows * cols;
  b->mat.assign(rm, rm + rows * cols);
  order_.push_back(b->name);
  bindings_[b->name] = std::move(b);
}

void Runner::bind_scalar(const char *name, int dtype, const double *bound) {
  check_new(*this, bindings_, order_, name);
  auto b = std::make_unique<Binding>();
  b->name = name;
  b->dir = DGK_SCALAR;
  b->is_scalar = true;
  b->host_dtype = b->dev_dtype = dtype ? dtype : DGK_FLOAT64;
  dtype_size(b->dev_dtype);
  b->total_values = 1;
  if (bound) {
    b->scalar_bound = true;
    b->scalar_value = *bound;
  }
  order_.push_back(b->name);
  bindings_[b->name] = std::move(b);
}

static size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

void Runner::allocate() {
  if (allocated) throw Error(DGK_ERR_STATE, "device memory already allocated");
  if (bindings_.empty()) throw Error(DGK_ERR_STATE, "no bindings defined - call DefineBindings first");
  const int is = int_type == DGK_INT32 ? 4 : 8;
  for (const std::string &n : order_) {
    Binding &b = *bindings_[n];
    if (b.is_scalar) continue;
    const int64_t vs = dtype_size(b.dev_dtype);
    if (b.is_matrix) {
      b.dbytes = (size_t)(b.rows * b.cols * vs);
      continue;
    }
    // CalculateAlignedOffsetsAndSize (runner/builder/builder.go:113-159): offsets in values
    if (ktotal <= 0) throw Error(DGK_ERR_INVALID, "total K is zero");
    const int64_t bpe = b.total_values * vs / ktotal;
    b.values_per_elem = bpe / vs;
    b.offsets.assign(npart + 1, 0);
    if (b.total_values % ktotal != 0 && !b.partitioned) {
      // not a whole number of values per element: one unpartitioned block (every offset 0)
      b.values_per_elem = 0;
      b.offsets[npart] = b.total_values;
      b.dbytes = (size_t)(b.total_values * vs);
      continue;
    }
    int64_t cur = 0;
    for (int p = 0; p < npart; ++p) {
      if (cur % b.align) cur = (cur + b.align - 1) / b.align * b.align;
      b.offsets[p] = cur / vs;
      cur += K[p] * b.values_per_elem * vs;
    }
    if (cur % b.align) cur = (cur + b.align - 1) / b.align * b.align;
    b.offsets[npart] = cur / vs;
    b.dbytes = (size_t)(b.offsets[npart] * vs);
    if (b.partitioned && b.layout == DGK_LAYOUT_FLAT)
      for (int p = 0; p < npart; ++p)
        if (b.part_values[p] > K[p] * b.values_per_elem)
          throw Error(DGK_ERR_INVALID, "partition " + std::to_string(p) + " of " + b.name +
                                           " holds more values than its K[p] elements allow");
  }
  // pooled arena: data then `<name>_offsets`, each 256-byte aligned
  size_t total = 0;
  std::vector<std::pair<size_t, size_t>> at;
  for (const std::string &n : order_) {
    Binding &b = *bindings_[n];
    size_t d = 0, o = 0;
    if (!b.is_scalar) {
      d = total;
      total = round_up(total + std::max<size_t>(b.dbytes, 1), 256);
      if (!b.is_matrix) {
        o = total;
        total = round_up(total + (size_t)(npart + 1) * is, 256);
      }
    }
    at.push_back({d, o});
  }
  if (host_only) {
    allocated = true;
    return;
  }
  cuda_check(cudaMalloc(reinterpret_cast<void **>(&arena_), std::max<size_t>(total, 256)), "cudaMalloc(arena)");
  cuda_check(cudaMemsetAsync(arena_, 0, std::max<size_t>(total, 256), stream_), "memset arena");
  size_t i = 0;
  for (const std::string &n : order_) {
    Binding &b = *bindings_[n];
    const auto pos = at[i++];
    if (b.is_scalar) continue;
    b.dptr = arena_ + pos.first;
    if (b.is_matrix) {
      // column-major device storage (runner/runner.go:375-417)
      std::vector<char> buf(b.dbytes);
      for (int64_t r = 0; r < b.rows; ++r)
        for (int64_t c = 0; c < b.cols; ++c) {
          const double v = b.mat[(size_t)(r * b.cols + c)];
          const size_t k = (size_t)(c * b.rows + r);
          switch (b.dev_dtype) {
            case DGK_FLOAT32: reinterpret_cast<float *>(buf.data())[k] = (float)v; break;
            case DGK_INT32: reinterpret_cast<int32_t *>(buf.data())[k] = (int32_t)v; break;
            case DGK_INT64: reinterpret_cast<int64_t *>(buf.data())[k] = (int64_t)v; break;
            default: reinterpret_cast<double *>(buf.data())[k] = v;
          }
        }
      cuda_check(cudaMemcpyAsync(b.dptr, buf.data(), b.dbytes, cudaMemcpyHostToDevice, stream_), "upload matrix");
      cuda_check(cudaStreamSynchronize(stream_), "sync");
      continue;
    }
    b.doffsets = arena_ + pos.second;
    std::vector<char> ho((size_t)(npart + 1) * is);
    for (int p = 0; p <= npart; ++p) {
      if (is == 4) {
        int32_t v = (int32_t)b.offsets[p];
        std::memcpy(&ho[(size_t)p * 4], &v, 4);
      } else {
        std::memcpy(&ho[(size_t)p * 8], &b.offsets[p], 8);
      }
    }
    cuda_check(cudaMemcpyAsync(b.doffsets, ho.data(), ho.size(), cudaMemcpyHostToDevice, stream_), "offsets");
    cuda_check(cudaStreamSynchronize(stream_), "sync");
  }
  allocated = true;
}

void *Runner::scratch(size_t bytes) {
  if (bytes > scratch_bytes_) {
    if (scratch_) {
      cuda_check(cudaStreamSynchronize(stream_), "sync");
      cudaFree(scratch_);
      scratch_ = nullptr;
    }
    scratch_bytes_ = round_up(bytes, 1 << 20);
    cuda_check(cudaMalloc(&scratch_, scratch_bytes_), "cudaMalloc(scratch)");
  }
  return scratch_;
}

// One partition host -> device: direct copy when types and layout agree, else stage the raw host bytes in
// scratch and convert / transpose on the GPU.
void Runner::host_to_partition(Binding &b, int part, const char *host, int64_t nvals) {
  const int hs = dtype_size(b.host_dtype), ds = dtype_size(b.dev_dtype);
  char *dst = b.is_matrix ? b.dptr : b.dptr + (size_t)(b.offsets[part] * ds);
  const bool transpose = b.layout == DGK_LAYOUT_MATRIX || b.is_matrix;
  if (!transpose && b.host_dtype == b.dev_dtype) {
    cuda_check(cudaMemcpyAsync(dst, host, (size_t)(nvals * hs), cudaMemcpyHostToDevice, stream_), "H2D copy");
    return;
  }
  void *s = scratch((size_t)(nvals * hs));
  cuda_check(cudaMemcpyAsync(s, host, (size_t)(nvals * hs), cudaMemcpyHostToDevice, stream_), "H2D copy");
  if (transpose) {
    const int64_t rows = b.rows, cols = nvals / b.rows;
    launch_transpose_convert(s, b.host_dtype, dst, b.dev_dtype, rows, cols, true, stream_);
  } else {
    launch_convert(s, b.host_dtype, dst, b.dev_dtype, nvals, stream_);
  }
  cuda_check(cudaGetLastError(), "convert kernel");
}

void Runner::partition_to_host(Binding &b, int part, char *host, int64_t nvals) {
  const int hs = dtype_size(b.host_dtype), ds = dtype_size(b.dev_dtype);
  const char *src = b.is_matrix ? b.dptr : b.dptr + (size_t)(b.offsets[part] * ds);
  const bool transpose = b.layout == DGK_LAYOUT_MATRIX || b.is_matrix;
  if (!transpose && b.host_dtype == b.dev_dtype) {
    cuda_check(cudaMemcpyAsync(host, src, (size_t)(nvals * hs), cudaMemcpyDeviceToHost, stream_), "D2H copy");
    return;
  }
  void *s = scratch((size_t)(nvals * hs));
  if (transpose) {
    const int64_t rows = b.rows, cols = nvals / b.rows;
    launch_transpose_convert(src, b.dev_dtype, s, b.host_dtype, rows, cols, false, stream_);
  } else {
    launch_convert(src, b.dev_dtype, s, b.host_dtype, nvals, stream_);
  }
  cuda_check(cudaGetLastError(), "convert kernel");
  cuda_check(cudaMemcpyAsync(host, s, (size_t)(nvals * hs), cudaMemcpyDeviceToHost, stream_), "D2H copy");
}

static int64_t part_host_values(const Binding &b, int p, int npart) {
  if (b.partitioned) return b.part_values[p];
  return npart == 1 || b.is_matrix ? b.total_values : 0;
}

void Runner::copy_to_device(const char *name, const void *host, int64_t bytes) {
  need_device(__func__);
  if (!allocated) throw Error(DGK_ERR_STATE, "device memory not allocated - call AllocateDevice first");
  Binding &b = binding(name);
  if (b.is_scalar) return;  // scalars travel by value (runner/memory_operations.go:52-55)
  if (!host) throw Error(DGK_ERR_INVALID, "null host pointer for " + b.name);
  const int hs = dtype_size(b.host_dtype);
  if (bytes != b.total_values * hs)
    throw Error(DGK_ERR_INVALID, "host size mismatch for " + b.name + ": got " + std::to_string(bytes) +
                                     " bytes, expected " + std::to_string(b.total_values * hs));
  const char *h = static_cast<const char *>(host);
  if (b.is_matrix || b.values_per_elem == 0 || (npart == 1 && !b.partitioned)) {
    host_to_partition(b, 0, h, b.total_values);
  } else {
    for (int p = 0; p < npart; ++p) {
      const int64_t nv = b.partitioned ? b.part_values[p] : K[p] * b.values_per_elem;
      host_to_partition(b, p, h, nv);
      h += nv * hs;
    }
  }
  cuda_check(cudaStreamSynchronize(stream_), "sync after H2D");
}

void Runner::copy_from_device(const char *name, void *host, int64_t bytes) {
  need_device(__func__);
  if (!allocated) throw Error(DGK_ERR_STATE, "device memory not allocated - call AllocateDevice first");
  Binding &b = binding(name);
  if (b.is_scalar) return;
  if (!host) throw Error(DGK_ERR_INVALID, "null host pointer for " + b.name);
  const int hs = dtype_size(b.host_dtype);
  if (bytes != b.total_values * hs)
    throw Error(DGK_ERR_INVALID, "host size mismatch for " + b.name + ": got " + std::to_string(bytes) +
                                     " bytes, expected " + std::to_string(b.total_values * hs));
  char *h = static_cast<char *>(host);
  if (b.is_matrix || b.values_per_elem == 0 || (npart == 1 && !b.partitioned)) {
    partition_to_host(b, 0, h, b.total_values);
  } else {
    for (int p = 0; p < npart; ++p) {
      const int64_t nv = b.partitioned ? b.part_values[p] : K[p] * b.values_per_elem;
      partition_to_host(b, p, h, nv);
      h += nv * hs;
    }
  }
  cuda_check(cudaStreamSynchronize(stream_), "sync after D2H");
}

void Runner::copy_partition_to_device(const char *name, int part, const void *host, int64_t bytes) {
  need_device(__func__);
  if (!allocated) throw Error(DGK_ERR_STATE, "device memory not allocated - call AllocateDevice first");
  Binding &b = binding(name);
  if (part < 0 || part >= npart) throw Error(DGK_ERR_INVALID, "invalid partition ID: " + std::to_string(part));
  if (b.is_scalar || b.is_matrix) throw Error(DGK_ERR_INVALID, b.name + " is not a partitioned array");
  const int64_t nv = b.partitioned ? b.part_values[part] : K[part] * b.values_per_elem;
  if (bytes != nv * dtype_size(b.host_dtype)) throw Error(DGK_ERR_INVALID, "partition size mismatch for " + b.name);
  host_to_partition(b, part, static_cast<const char *>(host), nv);
  cuda_check(cudaStreamSynchronize(stream_), "sync after H2D");
}

void Runner::copy_partition_from_device(const char *name, int part, void *host, int64_t bytes) {
  need_device(__func__);
  if (!allocated) throw Error(DGK_ERR_STATE, "device memory not allocated - call AllocateDevice first");
  Binding &b = binding(name);
  if (part < 0 || part >= npart) throw Error(DGK_ERR_INVALID, "invalid partition ID: " + std::to_string(part));
  if (b.is_scalar || b.is_matrix) throw Error(DGK_ERR_INVALID, b.name + " is not a partitioned array");
  // CopyPartitionToHost copies K[part] * values-per-element values (the reference copies only K[part]
  // values, runner/runner_copy.go:64-66 and :128-131; this backend copies the whole partition).
  const int64_t nv = b.partitioned ? b.part_values[part] : K[part] * b.values_per_elem;
  if (bytes != nv * dtype_size(b.host_dtype)) throw Error(DGK_ERR_INVALID, "partition size mismatch for " + b.name);
  partition_to_host(b, part, static_cast<char *>(host), nv);
  cuda_check(cudaStreamSynchronize(stream_), "sync after D2H");
}

void Runner::store_packed(Binding &b, const void *dsrc, int sdt) {
  if (b.is_scalar || b.is_matrix) throw Error(DGK_ERR_INVALID, b.name + " is not an array");
  const int ss = dtype_size(sdt), ds = dtype_size(b.dev_dtype);
  const char *src = static_cast<const char *>(dsrc);
  for (int p = 0; p < npart; ++p) {
    const int64_t nv = K[p] * b.values_per_elem;
    char *dst = b.dptr + (size_t)(b.offsets[p] * ds);
    if (sdt == b.dev_dtype)
      cuda_check(cudaMemcpyAsync(dst, src, (size_t)(nv * ss), cudaMemcpyDeviceToDevice, stream_), "D2D copy");
    else
      launch_convert(src, sdt, dst, b.dev_dtype, nv, stream_);
    src += nv * ss;
  }
  cuda_check(cudaGetLastError(), "store_packed");
}

KernelConfig &Runner::config(const std::string &name) {
  auto it = configs_.find(name);
  if (it == configs_.end())
    throw Error(DGK_ERR_STATE, "kernel " + name + " not configured - use ConfigureKernel first");
  return it->second;
}

void Runner::configure_kernel(const char *kname, int n, const char *const *params, const uint32_t *actions) {
  if (!allocated) throw Error(DGK_ERR_STATE, "device memory not allocated - call AllocateDevice first");
  KernelConfig cfg;
  cfg.name = kname;
  for (int i = 0; i < n; ++i) {
    Binding *b = find(params[i]);
    if (!b) throw Error(DGK_ERR_NOT_FOUND, "parameter configuration has no binding (" + std::string(params[i]) + ")");
    cfg.params.push_back({b, actions ? actions[i] : 0u});
  }
  configs_[kname] = std::move(cfg);
}

void Runner::build_kernel(const char *kname, const char *op_id) {
  need_device(__func__);
  KernelConfig &cfg = config(kname);
  cfg.op = make_op(*this, cfg, op_id ? op_id : kname);
}

void Runner::validate_offsets(const char *context) {
  const int is = int_type == DGK_INT32 ? 4 : 8;
  for (auto &kv : bindings_) {
    Binding &b = *kv.second;
    if (!b.doffsets) continue;
    std::vector<char> h((size_t)(npart + 1) * is);
    cuda_check(cudaMemcpyAsync(h.data(), b.doffsets, h.size(), cudaMemcpyDeviceToHost, stream_), "read offsets");
    cuda_check(cudaStreamSynchronize(stream_), "sync");
    for (int p = 0; p <= npart; ++p) {
      int64_t v = 0;
      if (is == 4) {
        int32_t w;
        std::memcpy(&w, &h[(size_t)p * 4], 4);
        v = w;
      } else {
        std::memcpy(&v, &h[(size_t)p * 8], 8);
      }
      if (v != b.offsets[p])
        throw Error(DGK_ERR_STATE, "OFFSET CORRUPTION DETECTED for " + b.name + " " + context + ": offset[" +
                                       std::to_string(p) + "] expected " + std::to_string(b.offsets[p]) + ", got " +
                                       std::to_string(v));
    }
  }
}

void Runner::check_status(const char *what) {
  int st = 0;
  cuda_check(cudaMemcpyAsync(&st, dstatus_, sizeof(int), cudaMemcpyDeviceToHost, stream_), "read status");
  cuda_check(cudaStreamSynchronize(stream_), "sync");
  if (st != 0) {
    cuda_check(cudaMemsetAsync(dstatus_, 0, sizeof(int), stream_), "reset status");
    throw Error(st == kStatusTimeoutCode ? DGK_ERR_TIMEOUT : DGK_ERR_INVALID,
                std::string(what) + ": device status word " + std::to_string(st) +
                    (st == 1 ? " (face gather index out of range)" : ""));
  }
}

// Scalar resolution (runner/kernel_execution.go:114-138): bound scalars win over explicit values (with the
// reference's warning), explicit values are taken in configuration order, and the result is ordered as the
// operator consumes them.
static std::vector<double> resolve_scalars(KernelConfig &cfg, int nscalars, const double *scalars) {
  std::map<std::string, double> sv;
  int sidx = 0;
  for (auto &pu : cfg.params) {
    if (!pu.b->is_scalar) continue;
    if (pu.b->scalar_bound) {
      if (sidx < nscalars && scalars[sidx] != pu.b->scalar_value)
        std::fprintf(stderr, "dgk: WARNING scalar %s is bound to %g; the explicit value %g is ignored\n",
                     pu.b->name.c_str(), pu.b->scalar_value, scalars[sidx]);
      sv[pu.b->name] = pu.b->scalar_value;
    } else if (sidx < nscalars) {
      sv[pu.b->name] = scalars[sidx];
    }
    ++sidx;
  }
  std::vector<double> vals;
  for (const std::string &s : cfg.op->scalar_names()) {
    auto f = sv.find(s);
    if (f == sv.end()) throw Error(DGK_ERR_INVALID, "scalar " + s + " not provided");
    vals.push_back(f->second);
  }
  return vals;
}

void Runner::execute_kernel(const char *kname, int nscalars, const double *scalars, void *const *host_ptrs) {
  auto it = configs_.find(kname);
  if (it == configs_.end())
    throw Error(DGK_ERR_STATE, "kernel " + std::string(kname) + " not configured - use ConfigureKernel first");
  KernelConfig &cfg = it->second;
  need_device(__func__);
  if (!cfg.op) throw Error(DGK_ERR_STATE, "kernel " + std::string(kname) + " not compiled - use BuildKernel first");
  if (validate_) validate_offsets((std::string("before kernel ") + kname).c_str());
  // pre-kernel copies (CopyTo)
  for (size_t i = 0; i < cfg.params.size(); ++i)
    if ((cfg.params[i].actions & DGK_COPY_TO) && host_ptrs && host_ptrs[i]) {
      Binding &b = *cfg.params[i].b;
      if (b.is_scalar) continue;
      copy_to_device(b.name.c_str(), host_ptrs[i], b.total_values * dtype_size(b.host_dtype));
    }
  std::vector<double> vals = resolve_scalars(cfg, nscalars, scalars);
  cfg.op->launch(*this, vals);
  cuda_check(cudaGetLastError(), "kernel launch");
  if (validate_) validate_offsets((std::string("after kernel ") + kname).c_str());
  bool back = false;
  for (size_t i = 0; i < cfg.params.size(); ++i)
    if ((cfg.params[i].actions & DGK_COPY_BACK) && host_ptrs && host_ptrs[i]) {
      Binding &b = *cfg.params[i].b;
      if (b.is_scalar) continue;
      copy_from_device(b.name.c_str(), host_ptrs[i], b.total_values * dtype_size(b.host_dtype));
      back = true;
    }
  if (back) check_status(kname);
}

Runner::Graph::~Graph() {
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
}

// Capture nlaunch launches of one built kernel, launch l with scalars[l*nscalars ...], into one CUDA graph.
// Operators that alternate ping-pong buffers swap them once per launch, so the count must be even for the
// buffers named by the bindings to hold the newest state after every replay.  The launches are recorded, not
// run: the state advances only when the graph is launched.
Runner::Graph *Runner::capture_graph(const char *kname, int nlaunch, int nscalars, const double *scalars) {
  need_device(__func__);
  KernelConfig &cfg = config(kname);
  if (!cfg.op) throw Error(DGK_ERR_STATE, "kernel " + std::string(kname) + " not compiled - use BuildKernel first");
  if (nlaunch < 2 || nlaunch % 2)
    throw Error(DGK_ERR_INVALID, "a captured sequence holds an even number (>= 2) of launches");
  if (nscalars < 0 || (nscalars > 0 && !scalars)) throw Error(DGK_ERR_INVALID, "scalar rows missing");
  for (auto &pu : cfg.params)
    if (!pu.b->is_scalar && (pu.actions & (DGK_COPY_TO | DGK_COPY_BACK)))
      throw Error(DGK_ERR_INVALID, "kernel " + std::string(kname) + ": a captured kernel carries no host copies");
  std::vector<std::vector<double>> rows;
  for (int l = 0; l < nlaunch; ++l) rows.push_back(resolve_scalars(cfg, nscalars, scalars + (size_t)l * nscalars));
  cfg.op->prepare(*this);
  cuda_check(cudaStreamSynchronize(stream_), "sync before capture");
  std::unique_ptr<Graph> g(new Graph);
  g->runner = this;
  g->nlaunch = nlaunch;
  cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
  try {
    for (int l = 0; l < nlaunch; ++l) cfg.op->launch(*this, rows[(size_t)l]);
  } catch (...) {
    cudaGraph_t tmp = nullptr;
    cudaStreamEndCapture(stream_, &tmp);
    if (tmp) cudaGraphDestroy(tmp);
    throw;
  }
  cuda_check(cudaStreamEndCapture(stream_, &g->graph), "cudaStreamEndCapture");
  cuda_check(cudaGraphInstantiate(&g->exec, g->graph, 0), "cudaGraphInstantiate");
  return g.release();
}

void Runner::launch_graph(Graph &g, int repeats) {
  need_device(__func__);
  if (g.runner != this) throw Error(DGK_ERR_INVALID, "graph belongs to another runner");
  for (int i = 0; i < repeats; ++i) cuda_check(cudaGraphLaunch(g.exec, stream_), "cudaGraphLaunch");
}

void Runner::sync() {
  need_device(__func__);
  cuda_check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
  check_status("sync");
}

std::string Runner::kernel_signature(const char *kname) {
  KernelConfig &cfg = config(kname);
  std::vector<std::string> args{"const int_t* K"};
  std::vector<Binding *> mats;
  for (auto &pu : cfg.params)
    if (pu.b->is_matrix && !pu.b->is_static) mats.push_back(pu.b);
  std::sort(mats.begin(), mats.end(), [](Binding *a, Binding *b) { return a->name < b->name; });
  for (Binding *m : mats) args.push_back(std::string("const ") + ctype(m->dev_dtype) + "* " + m->name);
  for (auto &pu : cfg.params) {
    Binding *b = pu.b;
    if (b->is_scalar || b->is_matrix) continue;
    const bool is_const = b->dir == DGK_INPUT;
    args.push_back(std::string(is_const ? "const " : "") + ctype(b->dev_dtype) + "* " + b->name + "_global");
    args.push_back("const int_t* " + b->name + "_offsets");
  }
  for (auto &pu : cfg.params)
    if (pu.b->is_scalar) args.push_back(std::string(ctype(pu.b->dev_dtype)) + " " + pu.b->name);
  std::string out;
  for (size_t i = 0; i < args.size(); ++i) out += (i ? ",\n\t" : "") + args[i];
  return out;
}

std::string Runner::preamble() {
  std::ostringstream s;
  s << "typedef " << (int_type == DGK_INT32 ? "int" : "long") << " int_t;\n\n";
  s << "#define NPART " << npart << "\n#define KpartMax " << kpart_max << "\n\n";
  std::vector<std::string> names;
  for (auto &kv : bindings_)
    if (!kv.second->is_scalar) names.push_back(kv.first);
  std::sort(names.begin(), names.end());
  bool any_static = false;
  for (auto &n : names) any_static |= bindings_[n]->is_matrix && bindings_[n]->is_static;
  char buf[64];
  if (any_static) {
    s << "// Static matrices\n";
    for (auto &n : names) {
      Binding &b = *bindings_[n];
      if (!(b.is_matrix && b.is_static)) continue;
      const bool f32 = b.dev_dtype == DGK_FLOAT32;
      s << "const " << (f32 ? "float " : "double ") << b.name << "[" << b.cols << "][" << b.rows << "] = {\n";
      for (int64_t j = 0; j < b.cols; ++j) {
        s << "  {";
        for (int64_t i = 0; i < b.rows; ++i) {
          const double v = b.mat[(size_t)(i * b.cols + j)];
          if (f32)
            std::snprintf(buf, sizeof buf, "%.8ff", v);
          else
            std::snprintf(buf, sizeof buf, "%.16e", v);
          s << buf << (i < b.rows - 1 ? ", " : "");
        }
        s << "}" << (j < b.cols - 1 ? "," : "") << "\n";
      }
      s << "};\n";
    }
    s << "\n";
  }
  s << "// Partition access macros\n";
  for (auto &n : names) {
    Binding &b = *bindings_[n];
    s << "#define " << n << "_PART(part) ((" << ctype(b.dev_dtype) << "*)(" << n << "_global + " << n
      << "_offsets[part]))\n";
  }
  s << "\n";
  for (int pass = 0; pass < 2; ++pass)
    for (auto &n : names) {
      Binding &b = *bindings_[n];
      if (!b.is_matrix || (pass == 0) != b.is_static) continue;
      const bool f32 = b.dev_dtype == DGK_FLOAT32;
      const std::string ty = f32 ? "float" : "double", zero = f32 ? "0.0f" : "0.0";
      const std::string term = b.is_static ? n + "[jj][ii]" : n + "[jj * " + std::to_string(b.rows) + " + ii]";
      for (int add = 0; add < 2; ++add) {
        s << "#define MATMUL_" << (add ? "ADD_" : "") << n << "(IN, OUT, K_VAL) {\\\n";
        s << "  for (int ii = 0; ii < " << b.rows << "; ++ii) {\\\n";
        s << "    for (int elem = 0; elem < KpartMax; ++elem; @inner) {\\\n";
        s << "      if (elem < (K_VAL)) {\\\n";
        s << "        " << ty << " sum = " << zero << ";\\\n";
        s << "        for (int jj = 0; jj < " << b.cols << "; ++jj) {\\\n";
        s << "          sum += " << term << " * (IN)[elem * " << b.cols << " + jj];\\\n";
        s << "        }\\\n";
        s << "        (OUT)[elem * " << b.rows << " + ii] " << (add ? "+=" : "=") << " sum;\\\n";
        s << "      }\\\n    }\\\n  }\\\n}\n\n";
      }
    }
  return s.str();
}

}  // namespace dgk
