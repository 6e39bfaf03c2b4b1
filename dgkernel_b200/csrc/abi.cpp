// extern "C" entry points of libdgk.so (declared in include/dgk.h).  Every call converts C++ exceptions
// into a status code plus a retrievable message; nothing throws across the ABI.
#include <cstring>
#include <memory>
#include <string>

#include "element.hpp"
#include "kernels.hpp"
#include "mesh.hpp"
#include "runner.hpp"

struct dgk_runner {
  dgk::Runner impl;
  dgk_runner(const int64_t *K, int n, int it, bool ho) : impl(K, n, it, ho) {}
};
struct dgk_element {
  dgk::RefElement impl;
  explicit dgk_element(int N) : impl(N) {}
};
struct dgk_graph {
  dgk_runner *r = nullptr;
  dgk::Runner::Graph *g = nullptr;
  ~dgk_graph() { delete g; }
};

namespace {
thread_local std::string g_error;

template <typename F>
int guard(dgk_runner *r, F &&f) {
  try {
    f();
    return DGK_OK;
  } catch (const dgk::Error &e) {
    (r ? r->impl.last_error : g_error) = e.what();
    return e.code;
  } catch (const std::invalid_argument &e) {
    (r ? r->impl.last_error : g_error) = e.what();
    return DGK_ERR_INVALID;
  } catch (const std::exception &e) {
    (r ? r->impl.last_error : g_error) = e.what();
    return DGK_ERR_INVALID;
  }
}

int copy_text(const std::string &s, char *buf, int64_t len) {
  if (!buf || len <= 0) return (int)std::min<size_t>(s.size() + 1, 0x7fffffff);
  const size_t n = std::min<size_t>(s.size(), (size_t)len - 1);
  std::memcpy(buf, s.data(), n);
  buf[n] = 0;
  return DGK_OK;
}
}  // namespace

void dgk::set_global_error(const std::string &msg) { g_error = msg; }

extern "C" {

int dgk_runner_create(const int64_t *K, int32_t npart, int32_t int_type, dgk_runner **out) {
  return guard(nullptr, [&] {
    if (!out) throw dgk::Error(DGK_ERR_INVALID, "null output pointer");
    *out = nullptr;
    *out = new dgk_runner(K, npart, int_type, false);
  });
}

int dgk_runner_create_host_only(const int64_t *K, int32_t npart, int32_t int_type, dgk_runner **out) {
  return guard(nullptr, [&] {
    if (!out) throw dgk::Error(DGK_ERR_INVALID, "null output pointer");
    *out = nullptr;
    *out = new dgk_runner(K, npart, int_type, true);
  });
}

int dgk_runner_free(dgk_runner *r) {
  delete r;
  return DGK_OK;
}

const char *dgk_last_error(const dgk_runner *r) { return r ? r->impl.last_error.c_str() : g_error.c_str(); }
const char *dgk_global_error(void) { return g_error.c_str(); }

int dgk_set_stream(dgk_runner *r, void *s) {
  return guard(r, [&] { r->impl.set_stream(static_cast<cudaStream_t>(s)); });
}
int dgk_sync(dgk_runner *r) {
  return guard(r, [&] { r->impl.sync(); });
}

int dgk_bind_array(dgk_runner *r, const char *name, int32_t dir, int32_t hdt, int32_t ddt, int64_t total,
                   int32_t part_count, const int64_t *part_values, int32_t align, int32_t layout, int64_t rows,
                   int64_t cols) {
  return guard(r, [&] { r->impl.bind_array(name, dir, hdt, ddt, total, part_count, part_values, align, layout, rows, cols); });
}
int dgk_bind_matrix(dgk_runner *r, const char *name, int64_t rows, int64_t cols, const double *rm, int32_t is_static,
                    int32_t ddt) {
  return guard(r, [&] { r->impl.bind_matrix(name, rows, cols, rm, is_static, ddt); });
}
int dgk_bind_scalar(dgk_runner *r, const char *name, int32_t dtype, const double *bound) {
  return guard(r, [&] { r->impl.bind_scalar(name, dtype, bound); });
}
int dgk_allocate(dgk_runner *r) {
  return guard(r, [&] { r->impl.allocate(); });
}

int dgk_copy_to_device(dgk_runner *r, const char *name, const void *host, int64_t bytes) {
  return guard(r, [&] { r->impl.copy_to_device(name, host, bytes); });
}
int dgk_copy_from_device(dgk_runner *r, const char *name, void *host, int64_t bytes) {
  return guard(r, [&] { r->impl.copy_from_device(name, host, bytes); });
}
int dgk_copy_partition_to_device(dgk_runner *r, const char *name, int32_t part, const void *host, int64_t bytes) {
  return guard(r, [&] { r->impl.copy_partition_to_device(name, part, host, bytes); });
}
int dgk_copy_partition_from_device(dgk_runner *r, const char *name, int32_t part, void *host, int64_t bytes) {
  return guard(r, [&] { r->impl.copy_partition_from_device(name, part, host, bytes); });
}
int dgk_copy_raw_from_device(dgk_runner *r, const char *name, int64_t value_offset, void *host, int64_t bytes) {
  return guard(r, [&] {
    dgk::Runner &R = r->impl;
    R.need_device("dgk_copy_raw_from_device");
    dgk::Binding &b = R.binding(name);
    if (b.is_scalar) throw dgk::Error(DGK_ERR_INVALID, b.name + " is a scalar");
    const int64_t es = dgk::dtype_size(b.dev_dtype);
    if (value_offset < 0 || bytes < 0 || (size_t)(value_offset * es + bytes) > b.dbytes)
      throw dgk::Error(DGK_ERR_INVALID, "raw read outside " + b.name);
    dgk::cuda_check(cudaMemcpyAsync(host, b.dptr + value_offset * es, (size_t)bytes, cudaMemcpyDeviceToHost,
                                    R.stream()), "D2H raw copy");
    dgk::cuda_check(cudaStreamSynchronize(R.stream()), "sync");
  });
}

int dgk_get_offsets(dgk_runner *r, const char *name, int64_t *out) {
  return guard(r, [&] {
    dgk::Binding &b = r->impl.binding(name);
    if (b.offsets.empty()) throw dgk::Error(DGK_ERR_INVALID, b.name + " has no partition offsets");
    std::memcpy(out, b.offsets.data(), sizeof(int64_t) * b.offsets.size());
  });
}
int dgk_device_ptr(dgk_runner *r, const char *name, void **out) {
  return guard(r, [&] {
    dgk::Binding &b = r->impl.binding(name);
    if (!r->impl.allocated) throw dgk::Error(DGK_ERR_STATE, "device memory not allocated");
    *out = b.dptr;
  });
}

int dgk_configure_kernel(dgk_runner *r, const char *kname, int32_t n, const char *const *params,
                         const uint32_t *actions) {
  return guard(r, [&] { r->impl.configure_kernel(kname, n, params, actions); });
}
int dgk_build_kernel(dgk_runner *r, const char *kname, const char *op_id) {
  return guard(r, [&] { r->impl.build_kernel(kname, op_id); });
}
int dgk_execute_kernel(dgk_runner *r, const char *kname, int32_t nscalars, const double *scalars,
                       void *const *host_ptrs) {
  return guard(r, [&] { r->impl.execute_kernel(kname, nscalars, scalars, host_ptrs); });
}
int dgk_kernel_signature(dgk_runner *r, const char *kname, char *buf, int64_t buflen) {
  int rc = DGK_OK;
  const int g = guard(r, [&] { rc = copy_text(r->impl.kernel_signature(kname), buf, buflen); });
  return g != DGK_OK ? g : rc;
}
int dgk_generate_preamble(dgk_runner *r, char *buf, int64_t buflen) {
  int rc = DGK_OK;
  const int g = guard(r, [&] { rc = copy_text(r->impl.preamble(), buf, buflen); });
  return g != DGK_OK ? g : rc;
}

int dgk_element_create(int32_t N, dgk_element **out) {
  return guard(nullptr, [&] { *out = new dgk_element(N); });
}
int dgk_element_free(dgk_element *e) {
  delete e;
  return DGK_OK;
}
int dgk_element_dims(const dgk_element *e, int32_t *Np, int32_t *Nfp) {
  if (!e) return DGK_ERR_INVALID;
  if (Np) *Np = e->impl.Np;
  if (Nfp) *Nfp = e->impl.Nfp;
  return DGK_OK;
}
int dgk_element_get(const dgk_element *e, const char *what, double *out, int64_t count) {
  return guard(nullptr, [&] {
    const dgk::RefElement &E = e->impl;
    const std::string w = what ? what : "";
    const std::vector<double> *v = w == "r"      ? &E.r
                                   : w == "s"    ? &E.s
                                   : w == "t"    ? &E.t
                                   : w == "V"    ? &E.V
                                   : w == "Vinv" ? &E.Vinv
                                   : w == "MassMatrix" ? &E.MassMatrix
                                   : w == "M"    ? &E.M
                                   : w == "Minv" ? &E.Minv
                                   : w == "Dr"   ? &E.Dr
                                   : w == "Ds"   ? &E.Ds
                                   : w == "Dt"   ? &E.Dt
                                   : w == "LIFT" ? &E.LIFT
                                                 : nullptr;
    if (!v) throw dgk::Error(DGK_ERR_NOT_FOUND, "unknown element array " + w);
    if (count != (int64_t)v->size())
      throw dgk::Error(DGK_ERR_INVALID, "element array " + w + " has " + std::to_string(v->size()) + " values");
    std::memcpy(out, v->data(), sizeof(double) * v->size());
  });
}
int dgk_element_fmask(const dgk_element *e, int32_t *out) {
  if (!e || !out) return DGK_ERR_INVALID;
  for (size_t i = 0; i < e->impl.Fmask.size(); ++i) out[i] = e->impl.Fmask[i];
  return DGK_OK;
}

int dgk_kuhn_mesh(int32_t n, int32_t nslab, double lo, double hi, double *VX, double *VY, double *VZ, int64_t *EToV,
                  int64_t *EToVp, int64_t *EToP) {
  return guard(nullptr, [&] { dgk::kuhn_mesh(n, nslab, lo, hi, VX, VY, VZ, EToV, EToVp, EToP); });
}
int dgk_ti_connect3d(int64_t K, const int64_t *EToV, int64_t *EToE, int64_t *EToF) {
  return guard(nullptr, [&] { dgk::ti_connect3d(K, EToV, EToE, EToF); });
}
int dgk_read_gambit(const char *path, int64_t *counts, double *VX, double *VY, double *VZ, int64_t *EToV,
                    int64_t *EToP, int64_t *bfaces) {
  return guard(nullptr, [&] {
    if (!path || !counts) throw dgk::Error(DGK_ERR_INVALID, "read gambit: null path or counts");
    const dgk::GambitMesh m = dgk::read_gambit(path);
    const int64_t nv = (int64_t)m.VX.size(), ne = (int64_t)m.EToV.size() / 4;
    counts[0] = nv;
    counts[1] = ne;
    counts[2] = (int64_t)m.bfaces.size();
    counts[3] = m.EToP.empty() ? 0 : 1;
    if (VX && VY && VZ)
      for (int64_t i = 0; i < nv; ++i) {
        VX[i] = m.VX[(size_t)i];
        VY[i] = m.VY[(size_t)i];
        VZ[i] = m.VZ[(size_t)i];
      }
    if (EToV) std::copy(m.EToV.begin(), m.EToV.end(), EToV);
    if (EToP && !m.EToP.empty()) std::copy(m.EToP.begin(), m.EToP.end(), EToP);
    if (bfaces)
      for (size_t i = 0; i < m.bfaces.size(); ++i) {
        bfaces[3 * i] = m.bfaces[i].elem;
        bfaces[3 * i + 1] = m.bfaces[i].face;
        bfaces[3 * i + 2] = m.bfaces[i].set;
      }
  });
}

int dgk_face_connector(int64_t K, int32_t Nfaces, int32_t Nfp, int32_t Np, const int64_t *vmapP, const int64_t *EToP,
                       int32_t npart, int64_t *pick_len, int64_t *pick_idx, int64_t *place_idx) {
  return guard(nullptr, [&] {
    dgk::FaceConnector fc = dgk::face_connector(K, Nfaces, Nfp, Np, vmapP, EToP, npart);
    const int P = fc.nparts;
    for (int i = 0; i < P * P; ++i) pick_len[i] = (int64_t)fc.pick[i].size();
    if (!pick_idx || !place_idx) return;
    int64_t o = 0;
    for (int i = 0; i < P * P; ++i)
      for (int64_t v : fc.pick[i]) pick_idx[o++] = v;
    o = 0;
    for (int i = 0; i < P * P; ++i)
      for (int64_t v : fc.place[i]) place_idx[o++] = v;
  });
}
int dgk_halo_plan(int64_t K, int32_t Nfaces, int32_t Nfp, int32_t Np, const int64_t *vmapP, const int64_t *EToP,
                  int32_t npart, const int32_t *part_rank, int32_t nranks, int32_t rank, const int64_t *local_off,
                  int64_t *counts, int32_t *gmap, int64_t *send_idx, int64_t *send_count, int64_t *recv_count,
                  int64_t *recv_off) {
  return guard(nullptr, [&] {
    if (!vmapP || !EToP || !part_rank || !local_off || !counts) throw dgk::Error(DGK_ERR_INVALID, "halo plan: null argument");
    const dgk::HaloPlan hp = dgk::halo_plan(K, Nfaces, Nfp, Np, vmapP, EToP, npart, part_rank, nranks, rank, local_off);
    counts[0] = (int64_t)hp.gmap.size();
    counts[1] = hp.halo_values;
    counts[2] = (int64_t)hp.send_idx.size();
    if (!gmap) return;
    std::copy(hp.gmap.begin(), hp.gmap.end(), gmap);
    if (send_idx) std::copy(hp.send_idx.begin(), hp.send_idx.end(), send_idx);
    if (send_count) std::copy(hp.send_count.begin(), hp.send_count.end(), send_count);
    if (recv_count) std::copy(hp.recv_count.begin(), hp.recv_count.end(), recv_count);
    if (recv_off) std::copy(hp.recv_off.begin(), hp.recv_off.end(), recv_off);
  });
}

int dgk_face_gather_map(int64_t K, int32_t Nfaces, int32_t Nfp, int32_t Np, const int64_t *vmapP,
                        const int64_t *EToP, int32_t npart, const int64_t *node_off, int32_t *gmap) {
  return guard(nullptr, [&] { dgk::face_gather_map(K, Nfaces, Nfp, Np, vmapP, EToP, npart, node_off, gmap); });
}

int dgk_compact_faces(int32_t npart, const int64_t *K, const int64_t *node_off, const int64_t *face_off,
                      int32_t Np, int32_t Nfp, const int32_t *gmap, int32_t *conn_out, uint8_t *table_out,
                      int32_t table_cap, int32_t *ncodes_out) {
  return guard(nullptr, [&] {
    if (npart < 1 || !K || !node_off || !face_off || !gmap || !conn_out || !ncodes_out)
      throw dgk::Error(DGK_ERR_INVALID, "compact faces: null argument or npart < 1");
    std::vector<int64_t> sp((size_t)npart + 1, 0);
    for (int p = 0; p < npart; ++p) sp[(size_t)p + 1] = sp[(size_t)p] + dgk::slot_padded(K[p]);
    dgk::CompactFaces cf = dgk::compact_faces(npart, K, node_off, face_off, sp.data(), Np, Nfp, gmap);
    std::copy(cf.conn.begin(), cf.conn.end(), conn_out);
    *ncodes_out = cf.ncodes;
    if (cf.ncodes > table_cap) throw dgk::Error(DGK_ERR_INVALID, "compact faces: table_cap too small");
    if (table_out) std::copy(cf.table.begin(), cf.table.end(), table_out);
  });
}

int dgk_tile_halo(int32_t npart, const int64_t *K, const int64_t *node_off, int32_t Np, int32_t Nfp,
                  const int32_t *conn, int32_t max_elems, int32_t max_halo, int32_t halo_floats, int32_t identity_code,
                  int32_t align, int64_t *counts_out, int32_t *part_out, int64_t *first_out, int32_t *nelem_out,
                  int32_t *halo_off_out, int32_t *halo_list_out, uint32_t *tconn_out) {
  return guard(nullptr, [&] {
    if (npart < 1 || !K || !node_off || !conn || !counts_out)
      throw dgk::Error(DGK_ERR_INVALID, "tile halo: null argument or npart < 1");
    std::vector<int64_t> sp((size_t)npart + 1, 0);
    for (int p = 0; p < npart; ++p) sp[(size_t)p + 1] = sp[(size_t)p] + dgk::slot_padded(K[p]);
    dgk::TileHalo th;
    try {
      th = dgk::tile_halo(npart, K, node_off, sp.data(), Np, Nfp, conn, max_elems, max_halo, halo_floats,
                          identity_code, align);
    } catch (const std::runtime_error &ex) {
      throw dgk::Error(DGK_ERR_INVALID, ex.what());
    }
    counts_out[0] = (int64_t)th.nelem.size();
    counts_out[1] = (int64_t)th.halo_list.size() / 2;
    if (part_out) std::copy(th.part.begin(), th.part.end(), part_out);
    if (first_out) std::copy(th.first.begin(), th.first.end(), first_out);
    if (nelem_out) std::copy(th.nelem.begin(), th.nelem.end(), nelem_out);
    if (halo_off_out) std::copy(th.halo_off.begin(), th.halo_off.end(), halo_off_out);
    if (halo_list_out) std::copy(th.halo_list.begin(), th.halo_list.end(), halo_list_out);
    if (tconn_out) std::copy(th.tconn.begin(), th.tconn.end(), tconn_out);
  });
}

int dgk_splitmix_uniform(uint64_t seed, int64_t count, double *out) {
  uint64_t s = seed;
  for (int64_t i = 0; i < count; ++i) out[i] = dgk::splitmix_uniform(s);
  return DGK_OK;
}

int dgk_setup_geometry(dgk_runner *r, const dgk_element *e, int64_t nverts, const double *VX, const double *VY,
                       const double *VZ, const int64_t *EToV, const int64_t *EToE, const int64_t *EToF, double period,
                       const char *const *names, double *hmin_out) {
  return guard(r, [&] {
    dgk::Runner &R = r->impl;
    if (!R.allocated) throw dgk::Error(DGK_ERR_STATE, "device memory not allocated - call AllocateDevice first");
    const dgk::RefElement &E = e->impl;
    const int64_t K = R.ktotal;
    cudaStream_t st = R.stream();
    std::vector<void *> owned;
    auto up = [&](const void *h, size_t bytes) {
      void *d = nullptr;
      dgk::cuda_check(cudaMalloc(&d, std::max<size_t>(bytes, 16)), "cudaMalloc(setup)");
      owned.push_back(d);
      dgk::cuda_check(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st), "upload setup");
      return d;
    };
    struct Free {
      std::vector<void *> &v;
      ~Free() {
        for (void *p : v) cudaFree(p);
      }
    } fr{owned};
    std::vector<double> rst(E.r);
    rst.insert(rst.end(), E.s.begin(), E.s.end());
    rst.insert(rst.end(), E.t.begin(), E.t.end());
    dgk::GeoSetup g{};
    g.N = E.N;
    g.Np = E.Np;
    g.Nfp = E.Nfp;
    g.K = K;
    g.VX = static_cast<const double *>(up(VX, sizeof(double) * nverts));
    g.VY = static_cast<const double *>(up(VY, sizeof(double) * nverts));
    g.VZ = static_cast<const double *>(up(VZ, sizeof(double) * nverts));
    g.EToV = static_cast<const int64_t *>(up(EToV, sizeof(int64_t) * 4 * K));
    g.EToE = EToE ? static_cast<const int64_t *>(up(EToE, sizeof(int64_t) * 4 * K)) : nullptr;
    g.EToF = EToF ? static_cast<const int64_t *>(up(EToF, sizeof(int64_t) * 4 * K)) : nullptr;
    g.rst = static_cast<const double *>(up(rst.data(), sizeof(double) * rst.size()));
    g.Dr = static_cast<const double *>(up(E.Dr.data(), sizeof(double) * E.Dr.size()));
    g.Ds = static_cast<const double *>(up(E.Ds.data(), sizeof(double) * E.Ds.size()));
    g.Dt = static_cast<const double *>(up(E.Dt.data(), sizeof(double) * E.Dt.size()));
    std::vector<int> fm(E.Fmask.begin(), E.Fmask.end());
    g.fmask = static_cast<const int *>(up(fm.data(), sizeof(int) * fm.size()));
    g.period = period;
    for (int64_t i = 0; i < 4 * K; ++i)
      if (EToV[i] < 0 || EToV[i] >= nverts) throw dgk::Error(DGK_ERR_INVALID, "EToV entry out of range");
    const int64_t nf = 4 * E.Nfp;
    double *buf = nullptr;
    dgk::cuda_check(cudaMalloc(reinterpret_cast<void **>(&buf), sizeof(double) * K * std::max<int64_t>(E.Np, nf)),
                    "cudaMalloc(setup field)");
    owned.push_back(buf);
    for (int w = 0; w < 18 && names; ++w) {
      if (!names[w]) continue;
      dgk::Binding &b = R.binding(names[w]);
      const int64_t vpe = w <= 12 ? E.Np : nf;
      if (b.values_per_elem != vpe)
        throw dgk::Error(DGK_ERR_INVALID, b.name + " must hold " + std::to_string(vpe) + " values per element");
      dgk::launch_geo_field(g, w, buf, st);
      R.store_packed(b, buf, DGK_FLOAT64);
    }
    if (names && (names[18] || names[19])) {
      if (!g.EToE || !g.EToF) throw dgk::Error(DGK_ERR_INVALID, "face maps need EToE and EToF");
      int64_t *mm = nullptr, *mp = nullptr;
      dgk::cuda_check(cudaMalloc(reinterpret_cast<void **>(&mm), sizeof(int64_t) * K * nf * 2), "cudaMalloc(maps)");
      owned.push_back(mm);
      mp = mm + K * nf;
      dgk::launch_build_maps(g, mm, mp, st);
      for (int w = 18; w < 20; ++w) {
        if (!names[w]) continue;
        dgk::Binding &b = R.binding(names[w]);
        if (b.values_per_elem != nf) throw dgk::Error(DGK_ERR_INVALID, b.name + " must hold 4*Nfp values per element");
        R.store_packed(b, w == 18 ? mm : mp, DGK_INT64);
      }
    }
    if (hmin_out) {
      const unsigned long long inf_bits = 0x7ff0000000000000ull;  // +inf: every distance is smaller
      unsigned long long *dm = static_cast<unsigned long long *>(up(&inf_bits, 8));
      dgk::launch_hmin(g, dm, st);
      unsigned long long h = 0;
      dgk::cuda_check(cudaMemcpyAsync(&h, dm, 8, cudaMemcpyDeviceToHost, st), "read hmin");
      dgk::cuda_check(cudaStreamSynchronize(st), "sync");
      double v;
      std::memcpy(&v, &h, 8);
      *hmin_out = v;
    }
    dgk::cuda_check(cudaStreamSynchronize(st), "sync setup");
  });
}

namespace {
// Evaluate the initial field per partition; modes_per_part selects one mode set per partition.
void init_field(dgk_runner *r, const char *name, const char *xn, const char *yn, const char *zn, int32_t kind,
                double mean, double amp, int32_t nmodes, const double *modes, bool modes_per_part) {
  dgk::Runner &R = r->impl;
  dgk::Binding &u = R.binding(name), &X = R.binding(xn), &Y = R.binding(yn), &Z = R.binding(zn);
  for (dgk::Binding *b : {&X, &Y, &Z})
    if (b->dev_dtype != u.dev_dtype || b->offsets != u.offsets)
      throw dgk::Error(DGK_ERR_INVALID, "coordinates must share the field's type and layout");
  if (nmodes < 0 || (nmodes > 0 && !modes)) throw dgk::Error(DGK_ERR_INVALID, "modes missing");
  const int64_t rows = (int64_t)nmodes * (modes_per_part ? R.npart : 1);
  double *dm = nullptr;
  if (rows > 0) {
    dgk::cuda_check(cudaMalloc(reinterpret_cast<void **>(&dm), sizeof(double) * 5 * rows), "cudaMalloc(modes)");
    dgk::cuda_check(cudaMemcpy(dm, modes, sizeof(double) * 5 * rows, cudaMemcpyHostToDevice), "modes");
  }
  for (int p = 0; p < R.npart; ++p) {
    const int64_t o = u.offsets[p], n = R.K[p] * u.values_per_elem;
    const double *mp = dm ? dm + (modes_per_part ? (int64_t)5 * nmodes * p : 0) : nullptr;
    if (u.dev_dtype == DGK_FLOAT64)
      dgk::launch_field<double>(reinterpret_cast<double *>(u.dptr) + o, reinterpret_cast<double *>(X.dptr) + o,
                                reinterpret_cast<double *>(Y.dptr) + o, reinterpret_cast<double *>(Z.dptr) + o, n, kind,
                                mean, amp, mp, nmodes, R.stream());
    else
      dgk::launch_field<float>(reinterpret_cast<float *>(u.dptr) + o, reinterpret_cast<float *>(X.dptr) + o,
                               reinterpret_cast<float *>(Y.dptr) + o, reinterpret_cast<float *>(Z.dptr) + o, n, kind,
                               mean, amp, mp, nmodes, R.stream());
  }
  dgk::cuda_check(cudaStreamSynchronize(R.stream()), "sync");
  if (dm) cudaFree(dm);
}
}  // namespace

int dgk_init_field(dgk_runner *r, const char *name, const char *xn, const char *yn, const char *zn, int32_t kind,
                   double mean, double amp, int32_t nmodes, const double *modes) {
  return guard(r, [&] { init_field(r, name, xn, yn, zn, kind, mean, amp, nmodes, modes, false); });
}

int dgk_init_field_parts(dgk_runner *r, const char *name, const char *xn, const char *yn, const char *zn,
                         double mean, int32_t nmodes, const double *modes) {
  return guard(r, [&] { init_field(r, name, xn, yn, zn, 2, mean, 0.0, nmodes, modes, true); });
}

int dgk_mlp_param_count(int32_t nin, int64_t *count) {
  return guard(nullptr, [&] {
    if (!count) throw dgk::Error(DGK_ERR_INVALID, "null output");
    *count = dgk::mlp_param_count(nin);
  });
}

int dgk_mlp_forward(const float *params, const float *X, int64_t n, int32_t nin, int32_t fp16, float *out,
                    void *half_scratch, void *cuda_stream) {
  return guard(nullptr, [&] {
    if (n < 0 || (n > 0 && (!params || !X || !out)) || (fp16 && !half_scratch))
      throw dgk::Error(DGK_ERR_INVALID, "mlp forward: null buffer or negative count");
    if (n == 0) return;
    dgk::launch_mlp_forward(params, X, n, nin, out, fp16, half_scratch, static_cast<cudaStream_t>(cuda_stream));
  });
}

int dgk_mlp_loss_grad(const float *params, const float *X, const float *y, int64_t n, int32_t nin, float *grad,
                      float *loss, void *cuda_stream) {
  return guard(nullptr, [&] {
    if (n <= 0 || !params || !X || !y || !grad || !loss)
      throw dgk::Error(DGK_ERR_INVALID, "mlp gradient: null buffer or no samples");
    dgk::launch_mlp_grad(params, X, y, n, nin, grad, loss, static_cast<cudaStream_t>(cuda_stream));
  });
}

int dgk_mlp_adam(float *params, const float *grad, float *m, float *v, int64_t count, float lr, float beta1,
                 float beta2, float eps, int32_t step, void *cuda_stream) {
  return guard(nullptr, [&] {
    if (count <= 0 || !params || !grad || !m || !v || step < 1)
      throw dgk::Error(DGK_ERR_INVALID, "adam: null buffer, empty parameter set or step < 1");
    dgk::launch_adam(params, grad, m, v, count, lr, beta1, beta2, eps, step, static_cast<cudaStream_t>(cuda_stream));
  });
}

int dgk_capture_graph(dgk_runner *r, const char *kernel_name, int32_t nlaunch, int32_t nscalars,
                      const double *scalars, dgk_graph **out) {
  return guard(r, [&] {
    if (!r || !out) throw dgk::Error(DGK_ERR_INVALID, "null runner or output");
    std::unique_ptr<dgk_graph> h(new dgk_graph);
    h->r = r;
    h->g = r->impl.capture_graph(kernel_name, nlaunch, nscalars, scalars);
    *out = h.release();
  });
}

int dgk_graph_launch(dgk_graph *g, int32_t repeats) {
  if (!g) {
    g_error = "null graph";
    return DGK_ERR_INVALID;
  }
  return guard(g->r, [&] { g->r->impl.launch_graph(*g->g, repeats); });
}

int dgk_graph_free(dgk_graph *g) {
  delete g;
  return DGK_OK;
}

}  // extern "C"
