// Named operators selected by BuildKernel (runner/runner.go:88-126): each resolves its roles against the
// kernel configuration, checks shapes and types once, and launches the precompiled sm_100a kernel.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <type_traits>

#include "kernels.hpp"
#include "mesh.hpp"
#include "runner.hpp"

namespace dgk {
namespace {

std::string lower(std::string s) {
  for (char &c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

// "name(k=v,k2=v2)" -> name, {k: v}
void parse_op(const std::string &id, std::string &name, std::map<std::string, std::string> &kv) {
  const size_t lp = id.find('(');
  name = id.substr(0, lp);
  if (lp == std::string::npos) return;
  const size_t rp = id.rfind(')');
  std::string body = id.substr(lp + 1, rp == std::string::npos ? std::string::npos : rp - lp - 1);
  size_t pos = 0;
  while (pos < body.size()) {
    size_t comma = body.find(',', pos);
    if (comma == std::string::npos) comma = body.size();
    const std::string item = body.substr(pos, comma - pos);
    const size_t eq = item.find('=');
    if (eq != std::string::npos) {
      auto trim = [](std::string s) {
        s.erase(0, s.find_first_not_of(" \t"));
        s.erase(s.find_last_not_of(" \t") + 1);
        return s;
      };
      kv[trim(item.substr(0, eq))] = trim(item.substr(eq + 1));
    }
    pos = comma + 1;
  }
}

struct Roles {
  KernelConfig &cfg;
  std::map<std::string, std::string> explicit_;
  std::string kname;

  Binding *array(const std::string &role, bool required = true) {
    auto it = explicit_.find(role);
    for (auto &pu : cfg.params) {
      Binding *b = pu.b;
      if (b->is_scalar || b->is_matrix) continue;
      if (it != explicit_.end() ? b->name == it->second : lower(b->name) == lower(role)) return b;
    }
    if (required)
      throw Error(DGK_ERR_NOT_FOUND, "kernel " + kname + ": no configured array for role '" + role + "'" +
                                         (it != explicit_.end() ? " (" + it->second + ")" : ""));
    return nullptr;
  }
  Binding *matrix(const std::string &role, bool required = true) {
    auto it = explicit_.find(role);
    for (auto &pu : cfg.params) {
      Binding *b = pu.b;
      if (!b->is_matrix) continue;
      if (it != explicit_.end()) {
        if (b->name == it->second) return b;
      } else if (b->name == role || b->name.rfind(role + "_", 0) == 0) {
        return b;
      }
    }
    if (required) throw Error(DGK_ERR_NOT_FOUND, "kernel " + kname + ": no configured matrix for role '" + role + "'");
    return nullptr;
  }
  int flag(const std::string &k, int dflt) {
    auto it = explicit_.find(k);
    return it == explicit_.end() ? dflt : std::atoi(it->second.c_str());
  }
  double num(const std::string &k, double dflt) {
    auto it = explicit_.find(k);
    return it == explicit_.end() ? dflt : std::atof(it->second.c_str());
  }
  std::string word(const std::string &k, const std::string &dflt) {
    auto it = explicit_.find(k);
    return it == explicit_.end() ? dflt : it->second;
  }
};

int order_from_np(int64_t np) {
  for (int n = 1; n <= 7; ++n)
    if ((n + 1) * (n + 2) * (n + 3) / 6 == np) return n;
  throw Error(DGK_ERR_UNSUPPORTED, "Np = " + std::to_string(np) + " is not a tetrahedron of order 1..7");
}

// Device buffer owned by an operator.
struct DevBuf {
  void *p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  template <typename T>
  T *get() const {
    return static_cast<T *>(p);
  }
  void upload(const void *h, size_t bytes) {
    alloc(bytes);
    cuda_check(cudaMemcpy(p, h, bytes, cudaMemcpyHostToDevice), "upload op buffer");
  }
  void alloc(size_t bytes) {
    if (p) cudaFree(p);
    p = nullptr;
    cuda_check(cudaMalloc(&p, std::max<size_t>(bytes, 16)), "cudaMalloc(op buffer)");
  }
};

template <typename T>
std::vector<T> cast(const std::vector<double> &v) {
  return std::vector<T>(v.begin(), v.end());
}

// Row-major rows x cols matrices (stacked) re-laid with rows padded to an even length, the layout the
// kernels' 16-byte pair loads require.
template <typename T>
std::vector<T> padded_rows(const std::vector<double> &v, int64_t rows, int64_t cols) {
  const int64_t ld = pad_even((int)cols), n = (int64_t)v.size() / cols;
  std::vector<T> out((size_t)(n * ld), T(0));
  for (int64_t r = 0; r < n; ++r)
    for (int64_t c = 0; c < cols; ++c) out[(size_t)(r * ld + c)] = (T)v[(size_t)(r * cols + c)];
  (void)rows;
  return out;
}

// Tile list over partitions: up to te consecutive elements of one partition per tile (the first nparts
// partitions; all when nparts < 0).
std::vector<Tile> make_tiles(const Runner &r, const Binding &node, const Binding *face, int te, int np, int nf,
                             int nparts = -1) {
  std::vector<Tile> t;
  for (int p = 0; p < (nparts < 0 ? r.npart : nparts); ++p)
    for (int64_t s = 0; s < r.K[p]; s += te) {
      Tile x;
      x.node_base = node.offsets[p] + s * np;
      x.face_base = face ? face->offsets[p] + s * nf : 0;
      x.nelem = (int32_t)std::min<int64_t>(te, r.K[p] - s);
      x.part = p;
      t.push_back(x);
    }
  return t;
}

void require(bool ok, const std::string &msg) {
  if (!ok) throw Error(DGK_ERR_INVALID, msg);
}

void same_layout(const Binding &a, const Binding &b, const std::string &what) {
  require(a.dev_dtype == b.dev_dtype, what + ": " + b.name + " must have the device type of " + a.name);
  require(a.values_per_elem == b.values_per_elem && a.offsets == b.offsets,
          what + ": " + b.name + " must share the partition layout of " + a.name);
}

// Volume derivative (`differentiate`) and the reference's volume-only computeRHS.
template <typename T>
struct DiffOp : Op {
  int N, mode, ntiles;
  Binding *u, *geo[9], *out[3];
  DevBuf dmat, tiles;
  DiffOp(Runner &r, Roles &R, int m) : mode(m) {
    static const char *gn[9] = {"Rx", "Ry", "Rz", "Sx", "Sy", "Sz", "Tx", "Ty", "Tz"};
    u = R.array(mode == 0 ? "U" : "u");
    for (int i = 0; i < 9; ++i) geo[i] = R.array(gn[i]);
    if (mode == 0) {
      out[0] = R.array("DuDx");
      out[1] = R.array("DuDy");
      out[2] = R.array("DuDz");
    } else {
      out[0] = R.array("rhsu");
      out[1] = out[2] = out[0];
    }
    Binding *Dr = R.matrix("Dr"), *Ds = R.matrix("Ds"), *Dt = R.matrix("Dt");
    const int64_t np = Dr->rows;
    N = order_from_np(np);
    require(u->values_per_elem == np, R.kname + ": " + u->name + " must hold Np values per element");
    for (Binding *b : geo) same_layout(*u, *b, R.kname);
    for (Binding *b : out) same_layout(*u, *b, R.kname);
    std::vector<double> d;
    for (Binding *m : {Dr, Ds, Dt}) {
      require(m->rows == np && m->cols == np, R.kname + ": " + m->name + " must be Np x Np");
      d.insert(d.end(), m->mat.begin(), m->mat.end());
    }
    auto dt = padded_rows<T>(d, 3 * np, np);
    dmat.upload(dt.data(), dt.size() * sizeof(T));
    auto tl = make_tiles(r, *u, nullptr, tile_elems(N), (int)np, 0);
    ntiles = (int)tl.size();
    tiles.upload(tl.data(), tl.size() * sizeof(Tile));
  }
  void launch(Runner &r, const std::vector<double> &) override {
    DiffArgs<T> A{};
    A.tiles = tiles.get<Tile>();
    A.ntiles = ntiles;
    A.u = reinterpret_cast<const T *>(u->dptr);
    for (int i = 0; i < 9; ++i) A.geo[i] = reinterpret_cast<const T *>(geo[i]->dptr);
    for (int i = 0; i < 3; ++i) A.out[i] = reinterpret_cast<T *>(out[i]->dptr);
    A.mode = mode;
    A.Dmat = dmat.get<T>();
    launch_diff<T>(N, A, r.num_sms, r.stream(), nullptr);
  }
};

// Fused strong-form Lax-Friedrichs RHS (+ LSERK4 stage).
template <typename T>
struct RhsOp : Op {
  int N, ntiles, rhs_only, conservative;
  Binding *u, *unext = nullptr, *resu = nullptr, *rhs = nullptr, *geo[9], *face[4], *gmap;
  DevBuf dmat, lift, fmask, tiles;
  // compact=1 (FP64): per-element geometry, compact connectivity and face-order table, each tile's first slot
  int compact = 0, ncodes = 0;
  DevBuf geoc, cconn, cftab, tslot;
  LaunchInfo info;
  RhsOp(Runner &r, Roles &R, int only) : rhs_only(only) {
    static const char *gn[9] = {"Rx", "Ry", "Rz", "Sx", "Sy", "Sz", "Tx", "Ty", "Tz"};
    static const char *fn[4] = {"nx", "ny", "nz", "Fscale"};
    conservative = R.flag("conservative", 0);
    compact = R.flag("compact", 0);
    // halo=1: the last partition holds neighbour values received from other ranks (slab exchange); it is read
    // through the gather map and never advanced
    const int halo = R.flag("halo", 0);
    require(halo == 0 || r.npart >= 2, R.kname + ": halo=1 needs a halo partition after the rank's own");
    const int tile_parts = r.npart - (halo ? 1 : 0);
    u = R.array("u");
    if (rhs_only) {
      rhs = R.array("rhs");
    } else {
      unext = R.array("uNext");
      resu = R.array("resu");
    }
    for (int i = 0; i < 9; ++i) geo[i] = R.array(gn[i]);
    for (int i = 0; i < 4; ++i) face[i] = R.array(fn[i]);
    gmap = R.array("gmap");
    Binding *Dr = R.matrix("Dr"), *Ds = R.matrix("Ds"), *Dt = R.matrix("Dt"), *L = R.matrix("LIFT"),
            *fm = R.matrix("Fmask");
    const int64_t np = Dr->rows;
    N = order_from_np(np);
    const int nfp = (N + 1) * (N + 2) / 2, nf = 4 * nfp;
    require(u->values_per_elem == np, R.kname + ": " + u->name + " must hold Np values per element");
    require(L->rows == np && L->cols == nf, R.kname + ": LIFT must be Np x 4Nfp");
    require(fm->rows * fm->cols == nf, R.kname + ": Fmask must hold 4*Nfp entries");
    for (Binding *b : geo) same_layout(*u, *b, R.kname);
    if (unext) same_layout(*u, *unext, R.kname);
    if (resu) same_layout(*u, *resu, R.kname);
    if (rhs) same_layout(*u, *rhs, R.kname);
    require(face[0]->values_per_elem == nf, R.kname + ": face arrays must hold 4*Nfp values per element");
    for (Binding *b : face) same_layout(*face[0], *b, R.kname);
    require(face[0]->dev_dtype == u->dev_dtype, R.kname + ": face arrays must have the state's device type");
    require(gmap->dev_dtype == DGK_INT32 && gmap->values_per_elem == nf && gmap->offsets == face[0]->offsets,
            R.kname + ": gmap must be int32 with the face arrays' layout");
    std::vector<double> d;
    for (Binding *m : {Dr, Ds, Dt}) {
      require(m->rows == np && m->cols == np, R.kname + ": " + m->name + " must be Np x Np");
      d.insert(d.end(), m->mat.begin(), m->mat.end());
    }
    auto dt = padded_rows<T>(d, 3 * np, np);
    dmat.upload(dt.data(), dt.size() * sizeof(T));
    auto lt = padded_rows<T>(L->mat, np, nf);
    lift.upload(lt.data(), lt.size() * sizeof(T));
    std::vector<int32_t> fmi(fm->mat.begin(), fm->mat.end());
    for (int32_t v : fmi) require(v >= 0 && v < np, R.kname + ": Fmask entry out of range");
    fmask.upload(fmi.data(), fmi.size() * sizeof(int32_t));
    // TMA-pipelined form when the order has one and every tile's streams start on 16-byte boundaries
    // (cp.async.bulk requirement); otherwise the register-staged form.
    // FP64: TMA streaming + element-local products on the FP64 tensor path; FP32: register-staged form.
    const char *no_tma = std::getenv("DGK_DISABLE_TMA");
    const bool tma_ok = !(no_tma && no_tma[0] == '1') && std::is_same<T, double>::value;
    const int te_tma = tma_ok ? dmma_tile_elems(N) : 0;
    use_tma = false;
    if (te_tma > 0) {
      auto tl = make_tiles(r, *u, face[0], te_tma, (int)np, nf, tile_parts);
      bool aligned = true;
      for (const Tile &x : tl)
        aligned = aligned && (x.node_base * (int64_t)sizeof(T)) % 16 == 0 &&
                  (x.face_base * (int64_t)sizeof(T)) % 16 == 0 && (x.face_base * 4) % 16 == 0;
      if (aligned) {
        use_tma = true;
        ntiles = (int)tl.size();
        tiles.upload(tl.data(), tl.size() * sizeof(Tile));
        if (compact) build_compact(r, R, tl, (int)np, nfp, tile_parts);
      }
    }
    if (compact && !use_tma)
      throw Error(DGK_ERR_UNSUPPORTED, R.kname + ": compact=1 is built for the FP64 tensor-path stage (orders 1..5, "
                                                 "16-byte aligned partitions)");
    if (!use_tma) {
      auto tl = make_tiles(r, *u, face[0], tile_elems(N), (int)np, nf, tile_parts);
      ntiles = (int)tl.size();
      tiles.upload(tl.data(), tl.size() * sizeof(Tile));
    }
  }
  bool use_tma = false;
  // The compact form's inputs, derived once from the bound arrays: the per-element geometry (checked
  // straight-sided), the gather map as neighbour bases and face-order codes, and each tile's first slot.
  void build_compact(Runner &r, Roles &R, const std::vector<Tile> &tl, int np, int nfp, int tile_parts) {
    const int P = r.npart;
    std::vector<int64_t> sp((size_t)P + 1, 0), ep((size_t)P + 1, 0);
    for (int p = 0; p < P; ++p) {
      sp[(size_t)p + 1] = sp[(size_t)p] + slot_padded(r.K[p]);
      ep[(size_t)p + 1] = ep[(size_t)p] + r.K[p];
    }
    const int64_t nslots = std::max<int64_t>(sp[(size_t)P], 1);
    {
      std::vector<double> z((size_t)(nslots * kCompactGeo64), 0.0);
      geoc.upload(z.data(), z.size() * sizeof(double));
    }
    DevBuf dep, dsp, dno, dfo, dbad;
    dep.upload(ep.data(), sizeof(int64_t) * (P + 1));
    dsp.upload(sp.data(), sizeof(int64_t) * P);
    dno.upload(geo[0]->offsets.data(), sizeof(int64_t) * P);
    dfo.upload(face[0]->offsets.data(), sizeof(int64_t) * P);
    int zero = 0;
    dbad.upload(&zero, sizeof(int));
    CompactGeoArgs<double> g{};
    g.npart = P;
    g.np = np;
    g.nf = 4 * nfp;
    g.elem_total = ep[(size_t)P];
    g.elem_prefix = dep.get<int64_t>();
    g.slot_prefix = dsp.get<int64_t>();
    g.node_off = dno.get<int64_t>();
    g.face_off = dfo.get<int64_t>();
    for (int i = 0; i < 9; ++i) g.geo[i] = reinterpret_cast<const double *>(geo[i]->dptr);
    for (int i = 0; i < 4; ++i) g.face[i] = reinterpret_cast<const double *>(face[i]->dptr);
    g.bad = dbad.get<int>();
    launch_compact_geo64(g, geoc.get<double>(), r.stream());
    int bad = 0;
    cuda_check(cudaMemcpyAsync(&bad, dbad.p, sizeof(int), cudaMemcpyDeviceToHost, r.stream()), "read affinity check");
    cuda_check(cudaStreamSynchronize(r.stream()), "compact geometry");
    if (bad)
      throw Error(DGK_ERR_UNSUPPORTED, R.kname + ": compact=1 needs straight-sided elements; " + std::to_string(bad) +
                                           " elements have metrics or face factors that vary by more than 1e-6");
    std::vector<int32_t> gm((size_t)gmap->offsets.back());
    cuda_check(cudaMemcpy(gm.data(), gmap->dptr, gm.size() * sizeof(int32_t), cudaMemcpyDeviceToHost), "read gmap");
    CompactFaces cf;
    try {
      cf = compact_faces(P, r.K.data(), u->offsets.data(), gmap->offsets.data(), sp.data(), np, nfp, gm.data());
    } catch (const std::exception &ex) {
      throw Error(DGK_ERR_INVALID, R.kname + ": " + ex.what());
    }
    ncodes = std::max(cf.ncodes, 1);
    if (cf.table.empty()) cf.table.assign((size_t)nfp, 0);
    cconn.upload(cf.conn.data(), std::max<size_t>(cf.conn.size(), 1) * sizeof(int32_t));
    cftab.upload(cf.table.data(), cf.table.size());
    std::vector<int64_t> ts(tl.size());
    for (size_t i = 0; i < tl.size(); ++i)
      ts[i] = sp[(size_t)tl[i].part] + (tl[i].node_base - u->offsets[(size_t)tl[i].part]) / np;
    tslot.upload(ts.data(), std::max<size_t>(ts.size(), 1) * sizeof(int64_t));
    (void)tile_parts;
  }
  std::vector<std::string> scalar_names() const override {
    if (rhs_only) return {};
    return {"a", "b", "dt"};
  }
  void launch(Runner &r, const std::vector<double> &s) override {
    RhsArgs<T> A{};
    A.tiles = tiles.get<Tile>();
    A.ntiles = ntiles;
    A.u_in = reinterpret_cast<const T *>(u->dptr);
    A.u_out = unext ? reinterpret_cast<T *>(unext->dptr) : nullptr;
    A.resu = resu ? reinterpret_cast<T *>(resu->dptr) : nullptr;
    A.rhs_out = rhs ? reinterpret_cast<T *>(rhs->dptr) : nullptr;
    for (int i = 0; i < 9; ++i) A.geo[i] = reinterpret_cast<const T *>(geo[i]->dptr);
    for (int i = 0; i < 4; ++i) A.face[i] = reinterpret_cast<const T *>(face[i]->dptr);
    A.gmap = reinterpret_cast<const int32_t *>(gmap->dptr);
    A.n_u_values = u->offsets.back();
    A.Dmat = dmat.get<T>();
    A.LIFT = lift.get<T>();
    A.fmask = fmask.get<int32_t>();
    if (!rhs_only) {
      A.a = (T)s[0];
      A.b = (T)s[1];
      A.dt = (T)s[2];
    }
    A.conservative = conservative;
    A.status = r.status_word();
    if (compact) {
      A.geoc = geoc.get<double>();
      A.conn = cconn.get<int32_t>();
      A.ftab = cftab.get<uint8_t>();
      A.ncodes = ncodes;
      A.tile_slot = tslot.get<int64_t>();
    }
    bool done = false;
    if constexpr (std::is_same<T, double>::value)
      if (use_tma) done = launch_rhs_dmma(N, A, rhs_only, r.num_sms, r.stream(), &info);
    if (!done) launch_rhs<T>(N, A, rhs_only, r.num_sms, r.stream(), &info);
    if (!rhs_only) std::swap(u->dptr, unext->dptr);  // "u" always names the newest state
  }
};

// Elementwise updates: the reference's updateSolution (mode 0) and the LSERK4 recurrence (mode 1).
template <typename T>
struct UpdateOp : Op {
  int mode, ntiles;
  int64_t np;
  Binding *u, *resu, *rhs;
  DevBuf tiles;
  UpdateOp(Runner &r, Roles &R, int m) : mode(m) {
    u = R.array("u");
    resu = R.array("resu");
    rhs = R.array(mode == 0 ? "rhsu" : "rhs");
    same_layout(*u, *resu, R.kname);
    same_layout(*u, *rhs, R.kname);
    np = std::max<int64_t>(1, u->values_per_elem);
    auto tl = make_tiles(r, *u, nullptr, 64, (int)np, 0);
    ntiles = (int)tl.size();
    tiles.upload(tl.data(), tl.size() * sizeof(Tile));
  }
  std::vector<std::string> scalar_names() const override {
    if (mode == 0) return {"rka", "rkb"};
    return {"a", "b", "dt"};
  }
  void launch(Runner &r, const std::vector<double> &s) override {
    launch_update<T>(tiles.get<Tile>(), ntiles, (int)np, reinterpret_cast<T *>(u->dptr),
                     reinterpret_cast<T *>(resu->dptr), reinterpret_cast<const T *>(rhs->dptr), s[0], s[1],
                     mode == 0 ? 0.0 : s[2], mode, r.num_sms, r.stream());
  }
};

// Generic MATMUL_<M>(IN, OUT, K[part]) / MATMUL_ADD_<M> (runner/builder/builder.go:355-410).
template <typename T>
struct MatmulOp : Op {
  int add, rows, cols;
  Binding *in, *out;
  DevBuf M, inoff, outoff, dK;
  int64_t kmax;
  MatmulOp(Runner &r, Roles &R, int a) : add(a) {
    Binding *m = R.matrix("M");
    in = R.array("IN");
    out = R.array("OUT");
    rows = (int)m->rows;
    cols = (int)m->cols;
    require(in->dev_dtype == out->dev_dtype, R.kname + ": IN and OUT must share a device type");
    require(in->values_per_elem == cols && out->values_per_elem == rows,
            R.kname + ": IN must hold cols and OUT rows values per element");
    auto mt = cast<T>(m->mat);
    M.upload(mt.data(), mt.size() * sizeof(T));
    inoff.upload(in->offsets.data(), sizeof(int64_t) * r.npart);
    outoff.upload(out->offsets.data(), sizeof(int64_t) * r.npart);
    dK.upload(r.K.data(), sizeof(int64_t) * r.npart);
    kmax = r.kpart_max;
  }
  void launch(Runner &r, const std::vector<double> &) override {
    launch_matmul<T>(M.get<T>(), rows, cols, reinterpret_cast<const T *>(in->dptr), reinterpret_cast<T *>(out->dptr),
                     inoff.get<int64_t>(), outoff.get<int64_t>(), dK.get<int64_t>(), r.npart, kmax, add, r.stream());
  }
};


// Mixed-precision stage (mixed.cu): compensated FP32 state (uhi + ulo), FP32 residual, compact affine
// geometry and compressed face maps, both derived here once from the per-node arrays and the gather map that
// the plain rhsStage reads.  Roles: uhi, ulo, uhiNext, uloNext, resu (float32 node arrays); Rx..Tz, nx, ny,
// nz, Fscale (float64 or float32, read at build time only); gmap (int32, value indices into uhi's layout);
// matrices Dr, Ds, Dt, LIFT, Fmask and Bary (Np x 4 barycentric coordinates of the nodes).
struct MixedOp : Op {
  int N = 0, ntiles = 0, conservative = 0, ncodes = 0, warps = 11, ring = 0, tensor = 0, mma = 0;
  Binding *uhi, *ulo, *uhin, *ulon, *resu;
  DevBuf tiles, geoE, conn, dm, lift, bary, vtx, ftab, fmask, amat, rexp, bmat;
  DevBuf tconn, hoff, hlist;  // tensor-core form: tile-local connectivity and the tiles' halo lists
  // learned-sensor viscosity (sensor=pp|mlp|mlp0 with mma=1)
  int lmode = 0;
  double eps0 = 1.0, s0 = 0.0, kappa = 1.0;
  float conf_lo = 0.1f, conf_hi = 0.9f;
  int64_t l_nslots = 0;
  Binding *geoB[9] = {}, *faceB[4] = {}, *gmapB = nullptr, *mlpB = nullptr;
  DevBuf l_dr, l_ds, l_dt, l_vinv, l_lift, l_top, l_hon, l_mlp16, l_sp, l_kp, l_uo, l_go, l_fo, l_eps, l_aslot, l_alist,
      l_tflag, l_vslot, l_tlist, l_counts, l_eq, l_visc;
  LaunchInfo info;

  template <typename G>
  void compact_geometry(Runner &r, Binding *const *geo, Binding *const *face, const std::vector<int64_t> &slot_prefix,
                        int np, int nf, const std::string &kname) {
    const int P = r.npart;
    std::vector<int64_t> ep(P + 1, 0);
    for (int p = 0; p < P; ++p) ep[p + 1] = ep[p] + r.K[p];
    DevBuf dep, dsp, dno, dfo, dbad;
    dep.upload(ep.data(), sizeof(int64_t) * (P + 1));
    dsp.upload(slot_prefix.data(), sizeof(int64_t) * P);
    dno.upload(geo[0]->offsets.data(), sizeof(int64_t) * P);
    dfo.upload(face[0]->offsets.data(), sizeof(int64_t) * P);
    int zero = 0;
    dbad.upload(&zero, sizeof(int));
    CompactGeoArgs<G> g{};
    g.npart = P;
    g.np = np;
    g.nf = nf;
    g.elem_total = ep[P];
    g.elem_prefix = dep.get<int64_t>();
    g.slot_prefix = dsp.get<int64_t>();
    g.node_off = dno.get<int64_t>();
    g.face_off = dfo.get<int64_t>();
    for (int i = 0; i < 9; ++i) g.geo[i] = reinterpret_cast<const G *>(geo[i]->dptr);
    for (int i = 0; i < 4; ++i) g.face[i] = reinterpret_cast<const G *>(face[i]->dptr);
    g.out = geoE.get<float>();
    g.bad = dbad.get<int>();
    launch_compact_geometry<G>(g, r.stream());
    int bad = 0;
    cuda_check(cudaMemcpyAsync(&bad, dbad.p, sizeof(int), cudaMemcpyDeviceToHost, r.stream()), "read affinity check");
    cuda_check(cudaStreamSynchronize(r.stream()), "compact geometry");
    if (bad)
      throw Error(DGK_ERR_UNSUPPORTED, kname + ": the mixed stage needs straight-sided elements; " + std::to_string(bad) +
                                           " elements have metrics or face factors that vary by more than 1e-6");
  }

  MixedOp(Runner &r, Roles &R) {
    static const char *gn[9] = {"Rx", "Ry", "Rz", "Sx", "Sy", "Sz", "Tx", "Ty", "Tz"};
    static const char *fn[4] = {"nx", "ny", "nz", "Fscale"};
    conservative = R.flag("conservative", 0);
    ring = R.flag("ring", 0);
    require(ring == 0 || (ring >= 2 && ring <= 24), R.kname + ": ring must be 0 (fill shared memory) or 2..24");
    uhi = R.array("uhi");
    ulo = R.array("ulo");
    uhin = R.array("uhiNext");
    ulon = R.array("uloNext");
    resu = R.array("resu");
    require(uhi->dev_dtype == DGK_FLOAT32, R.kname + ": uhi must be float32 on the device");
    for (Binding *b : {ulo, uhin, ulon, resu}) same_layout(*uhi, *b, R.kname);
    Binding *geo[9], *face[4];
    for (int i = 0; i < 9; ++i) geo[i] = R.array(gn[i]);
    for (int i = 0; i < 4; ++i) face[i] = R.array(fn[i]);
    Binding *gmap = R.array("gmap");
    Binding *Dr = R.matrix("Dr"), *Ds = R.matrix("Ds"), *Dt = R.matrix("Dt"), *L = R.matrix("LIFT"),
            *fm = R.matrix("Fmask"), *B = R.matrix("Bary");
    const int64_t np = Dr->rows;
    N = order_from_np(np);
    // orders 6 and 7 (and any order with tensor=1) run the precision form: exact integer-digit products on the
    // tensor cores
    tensor = R.flag("tensor", N >= 6 ? 1 : 0);
    if (tensor && !oz_supported(N))
      throw Error(DGK_ERR_UNSUPPORTED, R.kname + ": the tensor-core precision form is built for orders 4..7");
    if (!tensor && mixed_slot_bytes(N) == 0)
      throw Error(DGK_ERR_UNSUPPORTED, R.kname + ": the mixed stage is built for orders 1..5");
    // mma=1: the element-local products on the tensor cores with three-part BF16 operands (orders 1..4)
    mma = tensor ? 0 : R.flag("mma", 0);
    if (mma && !tcm_supported(N))
      throw Error(DGK_ERR_UNSUPPORTED, R.kname + ": the tensor-core mixed stage is built for orders 1..4");
    if (mma) {
      warps = R.flag("warps", 16);
      require(warps == 8 || warps == 16, R.kname + ": warps must be 8 or 16 with mma=1");
    } else {
      warps = R.flag("warps", 11);
      require(warps == 4 || warps == 8 || warps == 11, R.kname + ": warps must be 4, 8 or 11");
    }
    const int nfp = (N + 1) * (N + 2) / 2, nf = 4 * nfp;
    require(uhi->values_per_elem == np, R.kname + ": uhi must hold Np values per element");
    for (Binding *m : {Dr, Ds, Dt}) require(m->rows == np && m->cols == np, R.kname + ": " + m->name + " must be Np x Np");
    require(L->rows == np && L->cols == nf, R.kname + ": LIFT must be Np x 4Nfp");
    require(fm->rows * fm->cols == nf, R.kname + ": Fmask must hold 4*Nfp entries");
    require(B->rows == np && B->cols == 4, R.kname + ": Bary must be Np x 4");
    require(geo[0]->values_per_elem == np, R.kname + ": metric arrays must hold Np values per element");
    for (Binding *b : geo) same_layout(*geo[0], *b, R.kname);
    require(face[0]->values_per_elem == nf, R.kname + ": face arrays must hold 4*Nfp values per element");
    for (Binding *b : face) same_layout(*face[0], *b, R.kname);
    require(geo[0]->dev_dtype == face[0]->dev_dtype &&
                (geo[0]->dev_dtype == DGK_FLOAT64 || geo[0]->dev_dtype == DGK_FLOAT32),
            R.kname + ": metric and face arrays must share a float device type");
    require(gmap->dev_dtype == DGK_INT32 && gmap->values_per_elem == nf,
            R.kname + ": gmap must be int32 with 4*Nfp values per element");
    const int P = r.npart;
    std::vector<int64_t> slot_prefix(P + 1, 0);
    for (int p = 0; p < P; ++p) slot_prefix[p + 1] = slot_prefix[p] + slot_padded(r.K[p]);
    const int64_t nslots = std::max<int64_t>(slot_prefix[P], 1);
    {
      std::vector<float> z((size_t)(nslots * kMixedGeoWords), 0.f);
      geoE.upload(z.data(), z.size() * sizeof(float));
    }
    if (geo[0]->dev_dtype == DGK_FLOAT64)
      compact_geometry<double>(r, geo, face, slot_prefix, (int)np, nf, R.kname);
    else
      compact_geometry<float>(r, geo, face, slot_prefix, (int)np, nf, R.kname);
    // gather map -> neighbour base + face-order code per face (exact: the table reproduces every entry)
    std::vector<int32_t> gm((size_t)gmap->offsets.back());
    cuda_check(cudaMemcpy(gm.data(), gmap->dptr, gm.size() * sizeof(int32_t), cudaMemcpyDeviceToHost), "read gmap");
    CompactFaces cf;
    try {
      cf = compact_faces(P, r.K.data(), uhi->offsets.data(), gmap->offsets.data(), slot_prefix.data(), (int)np, nfp,
                         gm.data());
    } catch (const std::exception &ex) {
      throw Error(DGK_ERR_INVALID, R.kname + ": " + ex.what());
    }
    conn.upload(cf.conn.data(), std::max<size_t>(cf.conn.size(), 1) * sizeof(int32_t));
    TileHalo th;
    if (mma) {
      // tiles with their halos; a halo face's values arrive in the face's own point order: the identity row
      try {
        th = tile_halo(P, r.K.data(), uhi->offsets.data(), slot_prefix.data(), (int)np, nfp, cf.conn.data(),
                       tcm_tile_elems(), tcm_halo_capacity(), tcm_halo_floats(N), cf.ncodes, 4);
      } catch (const std::exception &ex) {
        throw Error(DGK_ERR_INVALID, R.kname + ": " + ex.what());
      }
      for (int i = 0; i < nfp; ++i) cf.table.push_back((uint8_t)i);
      ncodes = cf.ncodes + 1;
      tconn.upload(th.tconn.data(), std::max<size_t>(th.tconn.size(), 1) * sizeof(uint32_t));
      hoff.upload(th.halo_off.data(), th.halo_off.size() * sizeof(int32_t));
      th.halo_list.resize(std::max<size_t>(th.halo_list.size(), 4), 0);
      hlist.upload(th.halo_list.data(), th.halo_list.size() * sizeof(int32_t));
    } else {
      ncodes = std::max(cf.ncodes, 1);
      if (cf.table.empty()) cf.table.assign((size_t)nfp, 0);
    }
    ftab.upload(cf.table.data(), cf.table.size());
    // Dr, Ds, Dt interleaved by column pairs ([i][j/2][r,s,t][j%2]), columns padded to a multiple of 4 with
    // zeros: one row's pair of columns feeds three paired FMAs
    const int npj = ((int)np + 3) & ~3;
    std::vector<float> d((size_t)(np * npj * 3), 0.f);
    const Binding *D3[3] = {Dr, Ds, Dt};
    for (int64_t i = 0; i < np; ++i)
      for (int64_t j = 0; j < np; ++j)
        for (int c = 0; c < 3; ++c)
          d[(size_t)(i * 3 * npj + (j / 2) * 6 + c * 2 + (j % 2))] = (float)D3[c]->mat[(size_t)(i * np + j)];
    dm.upload(d.data(), d.size() * sizeof(float));
    auto lt = cast<float>(L->mat);
    lift.upload(lt.data(), lt.size() * sizeof(float));
    std::vector<double> bw((size_t)(np * 3));
    int32_t vt[4];
    for (int c = 0; c < 4; ++c) {
      int64_t best = 0;
      for (int64_t i = 0; i < np; ++i)
        if (B->mat[(size_t)(i * 4 + c)] > B->mat[(size_t)(best * 4 + c)]) best = i;
      require(std::fabs(B->mat[(size_t)(best * 4 + c)] - 1.0) < 1e-10, R.kname + ": Bary has no vertex node");
      vt[c] = (int32_t)best;
    }
    for (int64_t i = 0; i < np; ++i)
      for (int c = 0; c < 3; ++c) bw[(size_t)(i * 3 + c)] = B->mat[(size_t)(i * 4 + c + 1)];
    bary.upload(bw.data(), bw.size() * sizeof(double));
    vtx.upload(vt, sizeof(vt));
    std::vector<int32_t> fmi(fm->mat.begin(), fm->mat.end());
    for (int32_t v : fmi) require(v >= 0 && v < np, R.kname + ": Fmask entry out of range");
    fmask.upload(fmi.data(), fmi.size() * sizeof(int32_t));
    if (tensor) {  // integer digits of Dr, Ds, Dt and LIFT in 4 KB chunks, and their row exponents
      std::vector<uint8_t> packed;
      std::vector<int32_t> re;
      oz_pack_operands(N, Dr->mat.data(), Ds->mat.data(), Dt->mat.data(), L->mat.data(), packed, re);
      amat.upload(packed.data(), packed.size());
      rexp.upload(re.data(), re.size() * sizeof(int32_t));
    }
    if (mma) {
      std::vector<uint16_t> packed;
      tcm_pack_operands(N, Dr->mat.data(), Ds->mat.data(), Dt->mat.data(), L->mat.data(), packed);
      bmat.upload(packed.data(), packed.size() * sizeof(uint16_t));
    }
    const int te = tensor ? oz_tile_elems() : kMixedSlotElems;
    std::vector<MTile> tl;
    auto add_tile = [&](int p, int64_t s0, int64_t ne) {
      MTile x;
      x.node_base = uhi->offsets[p] + s0 * np;
      x.elem_slot = slot_prefix[p] + s0;
      x.nelem = (int32_t)ne;
      x.part = p;
      require((x.node_base * 4) % 16 == 0, R.kname + ": partition offsets of uhi must be 16-byte aligned");
      tl.push_back(x);
    };
    if (mma) {
      for (size_t i = 0; i < th.nelem.size(); ++i) add_tile(th.part[i], th.first[i], th.nelem[i]);
    } else {
      for (int p = 0; p < P; ++p)
        for (int64_t s0 = 0; s0 < r.K[p]; s0 += te) add_tile(p, s0, std::min<int64_t>(te, r.K[p] - s0));
    }
    ntiles = (int)tl.size();
    tiles.upload(tl.data(), std::max<size_t>(tl.size(), 1) * sizeof(MTile));
    const std::string sensor = lower(R.word("sensor", "none"));
    if (sensor != "none") {
      if (sensor == "pp") lmode = 1;
      else if (sensor == "mlp") lmode = 2;
      else if (sensor == "mlp0") lmode = 3;
      else throw Error(DGK_ERR_INVALID, R.kname + ": sensor must be none, pp, mlp or mlp0");
      require(mma && ls_supported(N), R.kname + ": the learned-sensor viscosity runs on the tensor-core mixed stage "
                                               "(mma=1, orders 1..4)");
      require(geo[0]->dev_dtype == DGK_FLOAT64 && face[0]->dev_dtype == DGK_FLOAT64,
              R.kname + ": the viscous term reads float64 metric and face arrays");
      eps0 = R.num("eps0", 1.0);
      kappa = R.num("kappa", 1.0);
      conf_lo = (float)R.num("lo", 0.1);
      conf_hi = (float)R.num("hi", 0.9);
      require(kappa > 0.0 && eps0 >= 0.0, R.kname + ": kappa > 0 and eps0 >= 0");
      s0 = -(R.num("c0", 0.0) + 4.0 * std::log10((double)N));
      for (int i = 0; i < 9; ++i) geoB[i] = geo[i];
      for (int i = 0; i < 4; ++i) faceB[i] = face[i];
      gmapB = gmap;
      Binding *Vi = R.matrix("Vinv");
      require(Vi->rows == np && Vi->cols == np, R.kname + ": Vinv must be Np x Np");
      auto rm = [&](const std::vector<double> &m, DevBuf &d) { d.upload(m.data(), m.size() * sizeof(double)); };
      // the sparse passes read Dr, Ds, Dt and LIFT transposed (column j contiguous over rows i)
      auto tr = [&](const std::vector<double> &m, int64_t rows, int64_t cols, DevBuf &d) {
        std::vector<double> t((size_t)(rows * cols));
        for (int64_t i = 0; i < rows; ++i)
          for (int64_t j = 0; j < cols; ++j) t[(size_t)(j * rows + i)] = m[(size_t)(i * cols + j)];
        d.upload(t.data(), t.size() * sizeof(double));
      };
      tr(Dr->mat, np, np, l_dr);
      tr(Ds->mat, np, np, l_ds);
      tr(Dt->mat, np, np, l_dt);
      rm(Vi->mat, l_vinv);
      tr(L->mat, np, nf, l_lift);
      if (lmode >= 2) {
        mlpB = R.matrix("MLP");
        require(mlpB->rows * mlpB->cols == mlp_param_count((int)np) && mlpB->dev_dtype == DGK_FLOAT32,
                R.kname + ": MLP must hold " + std::to_string(mlp_param_count((int)np)) + " float32 parameters");
        l_mlp16.alloc(sizeof(uint16_t) * ((size_t)mlp_param_count((int)np) + 8));
      }
      std::vector<int32_t> tp;
      for (int i = 0; i <= N; ++i)  // modes ordered i, j, k (vandermonde3d.go:15-42)
        for (int j = 0; j <= N - i; ++j)
          for (int k = 0; k <= N - i - j; ++k) tp.push_back(i + j + k == N ? 1 : 0);
      l_top.upload(tp.data(), tp.size() * sizeof(int32_t));
      // h_e / N per element slot, h_e = 2 / max Fscale over the element's face points
      l_nslots = slot_prefix[P];
      std::vector<double> fs((size_t)face[3]->offsets.back());
      cuda_check(cudaMemcpy(fs.data(), face[3]->dptr, fs.size() * sizeof(double), cudaMemcpyDeviceToHost), "Fscale");
      std::vector<double> h((size_t)std::max<int64_t>(l_nslots, 1), 0.0);
      for (int p = 0; p < P; ++p)
        for (int64_t e = 0; e < r.K[p]; ++e) {
          double m = 0.0;
          for (int k = 0; k < nf; ++k) m = std::max(m, fs[(size_t)(face[3]->offsets[p] + e * nf + k)]);
          require(m > 0.0, R.kname + ": Fscale must be positive");
          h[(size_t)(slot_prefix[p] + e)] = 2.0 / m / N;
        }
      l_hon.upload(h.data(), h.size() * sizeof(double));
      std::vector<int64_t> kp(r.K.begin(), r.K.end()), uo(uhi->offsets.begin(), uhi->offsets.begin() + P),
          go(geo[0]->offsets.begin(), geo[0]->offsets.begin() + P), fo(face[0]->offsets.begin(), face[0]->offsets.begin() + P);
      l_sp.upload(slot_prefix.data(), slot_prefix.size() * sizeof(int64_t));
      l_kp.upload(kp.data(), kp.size() * sizeof(int64_t));
      l_uo.upload(uo.data(), uo.size() * sizeof(int64_t));
      l_go.upload(go.data(), go.size() * sizeof(int64_t));
      l_fo.upload(fo.data(), fo.size() * sizeof(int64_t));
      const size_t ns = (size_t)std::max<int64_t>(l_nslots, 1);
      l_eps.alloc(ns * sizeof(double));
      std::vector<int32_t> minus((size_t)ns, -1), zero((size_t)ns, 0);
      l_aslot.upload(minus.data(), ns * sizeof(int32_t));
      l_vslot.upload(minus.data(), ns * sizeof(int32_t));
      l_tflag.upload(zero.data(), ns * sizeof(int32_t));
      l_alist.alloc(ns * sizeof(int32_t));
      l_tlist.alloc(ns * sizeof(int32_t));
      l_counts.alloc(4 * sizeof(int32_t));
      l_eq.alloc(ns * 3 * (size_t)np * sizeof(double));  // capacity: every element active
      l_visc.alloc(ns * (size_t)np * sizeof(double));
    }
  }
  // Learned-sensor viscosity of the current state: sensor, active and touched lists, BR1 gradient and
  // divergence on the GPU; the tensor-core stage then adds the viscous right-hand side.
  void launch_viscosity(Runner &r) {
    LsArgs L{};
    L.tiles = tiles.get<MTile>();
    L.ntiles = ntiles;
    L.npart = r.npart;
    L.slot_prefix = l_sp.get<int64_t>();
    L.kpart = l_kp.get<int64_t>();
    L.uoff = l_uo.get<int64_t>();
    L.goff = l_go.get<int64_t>();
    L.foff = l_fo.get<int64_t>();
    L.uhi = reinterpret_cast<const float *>(uhi->dptr);
    L.ulo = reinterpret_cast<const float *>(ulo->dptr);
    for (int i = 0; i < 9; ++i) L.geo[i] = reinterpret_cast<const double *>(geoB[i]->dptr);
    for (int i = 0; i < 4; ++i) L.face[i] = reinterpret_cast<const double *>(faceB[i]->dptr);
    L.gmap = reinterpret_cast<const int32_t *>(gmapB->dptr);
    L.conn = conn.get<int32_t>();
    L.n_u_values = uhi->offsets.back();
    L.Dr = l_dr.get<double>();
    L.Ds = l_ds.get<double>();
    L.Dt = l_dt.get<double>();
    L.Vinv = l_vinv.get<double>();
    L.LIFT = l_lift.get<double>();
    L.fmask = fmask.get<int32_t>();
    L.top = l_top.get<int32_t>();
    L.h_over_n = l_hon.get<double>();
    L.mode = lmode;
    L.eps0 = eps0;
    L.s0 = s0;
    L.kappa = kappa;
    L.conf_lo = conf_lo;
    L.conf_hi = conf_hi;
    if (lmode >= 2) {
      launch_to_half(reinterpret_cast<const float *>(mlpB->dptr), l_mlp16.p, mlp_param_count((N + 1) * (N + 2) * (N + 3) / 6), r.stream());
      L.mlp16 = l_mlp16.get<unsigned short>();
    }
    L.eps = l_eps.get<double>();
    L.aslot = l_aslot.get<int32_t>();
    L.alist = l_alist.get<int32_t>();
    L.tflag = l_tflag.get<int32_t>();
    L.vslot = l_vslot.get<int32_t>();
    L.tlist = l_tlist.get<int32_t>();
    L.counts = l_counts.get<int32_t>();
    L.eq = l_eq.get<double>();
    L.visc = l_visc.get<double>();
    L.nslots = l_nslots;
    L.status = r.status_word();
    launch_ls(N, L, r.num_sms, r.stream());
  }
  std::vector<std::string> scalar_names() const override { return {"a", "b", "dt"}; }
  void prepare(Runner &) override {
    if (lmode) prepare_ls(N);
    if (mma)
      prepare_rhs_tcm(N, warps);
    else if (tensor)
      prepare_rhs_oz(N);
    else
      prepare_rhs_mixed(N, warps);
  }
  void launch_tensor(Runner &r, const std::vector<double> &s) {
    OzArgs A{};
    A.tiles = tiles.get<MTile>();
    A.ntiles = ntiles;
    A.uhi_in = reinterpret_cast<const float *>(uhi->dptr);
    A.ulo_in = reinterpret_cast<const float *>(ulo->dptr);
    A.uhi_out = reinterpret_cast<float *>(uhin->dptr);
    A.ulo_out = reinterpret_cast<float *>(ulon->dptr);
    A.resu = reinterpret_cast<float *>(resu->dptr);
    A.geo = geoE.get<float>();
    A.conn = conn.get<int32_t>();
    A.n_u_values = uhi->offsets.back();
    A.amat = amat.get<unsigned char>();
    A.rexp = rexp.get<int32_t>();
    A.bary = bary.get<double>();
    A.vtx = vtx.get<int32_t>();
    A.ftab = ftab.get<uint8_t>();
    A.fmask = fmask.get<int32_t>();
    A.ncodes = ncodes;
    A.a = s[0];
    A.b = s[1];
    A.dt = s[2];
    A.status = r.status_word();
    if (!launch_rhs_oz(N, A, conservative, r.num_sms, r.stream(), &info))
      throw Error(DGK_ERR_UNSUPPORTED, "tensor-core precision stage: shared memory does not fit this order");
    std::swap(uhi->dptr, uhin->dptr);
    std::swap(ulo->dptr, ulon->dptr);
  }
  void launch(Runner &r, const std::vector<double> &s) override {
    if (ntiles == 0) return;
    if (tensor) return launch_tensor(r, s);
    MixedArgs A{};
    A.tiles = tiles.get<MTile>();
    A.ntiles = ntiles;
    A.uhi_in = reinterpret_cast<const float *>(uhi->dptr);
    A.ulo_in = reinterpret_cast<const float *>(ulo->dptr);
    A.uhi_out = reinterpret_cast<float *>(uhin->dptr);
    A.ulo_out = reinterpret_cast<float *>(ulon->dptr);
    A.resu = reinterpret_cast<float *>(resu->dptr);
    A.geo = geoE.get<float>();
    A.conn = conn.get<int32_t>();
    A.n_u_values = uhi->offsets.back();
    A.Dm = dm.get<float>();
    A.lift = lift.get<float>();
    A.bary = bary.get<double>();
    A.vtx = vtx.get<int32_t>();
    A.ftab = ftab.get<uint8_t>();
    A.fmask = fmask.get<int32_t>();
    A.ncodes = ncodes;
    A.a = (float)s[0];
    A.b = s[1];
    A.dt = (float)s[2];
    A.conservative = conservative;
    A.status = r.status_word();
    if (mma) {
      A.bmat = bmat.get<unsigned char>();
      A.conn = tconn.get<int32_t>();
      A.halo_off = hoff.get<int32_t>();
      A.halo_list = hlist.get<int32_t>();
      if (lmode) {
        launch_viscosity(r);
        A.vslot = l_vslot.get<int32_t>();
        A.visc = l_visc.get<double>();
      }
      if (!launch_rhs_tcm(N, A, warps, r.num_sms, r.stream(), &info))
        throw Error(DGK_ERR_UNSUPPORTED, "tensor-core mixed stage: shared memory does not fit this order");
      std::swap(uhi->dptr, uhin->dptr);
      std::swap(ulo->dptr, ulon->dptr);
      return;
    }
    if (!launch_rhs_mixed(N, A, warps, ring, r.num_sms, r.stream(), &info))
      throw Error(DGK_ERR_UNSUPPORTED, "mixed stage: no launch shape fits shared memory for this order");
    std::swap(uhi->dptr, uhin->dptr);  // "uhi"/"ulo" always name the newest state
    std::swap(ulo->dptr, ulon->dptr);
  }
};

// State split u (float64) -> uhi + ulo (float32 pair) and the join back, per partition.
struct SplitJoinOp : Op {
  int join;
  Binding *u, *hi, *lo;
  DevBuf cnt, uo, ho, lo_off;
  SplitJoinOp(Runner &r, Roles &R, int j) : join(j) {
    u = R.array("u");
    hi = R.array("uhi");
    lo = R.array("ulo");
    require(u->dev_dtype == DGK_FLOAT64, R.kname + ": u must be float64 on the device");
    require(hi->dev_dtype == DGK_FLOAT32, R.kname + ": uhi must be float32 on the device");
    same_layout(*hi, *lo, R.kname);
    require(u->values_per_elem == hi->values_per_elem, R.kname + ": u and uhi must hold the same values per element");
    std::vector<int64_t> c((size_t)r.npart);
    for (int p = 0; p < r.npart; ++p) c[(size_t)p] = r.K[p] * hi->values_per_elem;
    cnt.upload(c.data(), c.size() * sizeof(int64_t));
    uo.upload(u->offsets.data(), sizeof(int64_t) * r.npart);
    ho.upload(hi->offsets.data(), sizeof(int64_t) * r.npart);
    lo_off.upload(lo->offsets.data(), sizeof(int64_t) * r.npart);
  }
  void launch(Runner &r, const std::vector<double> &) override {
    SplitJoinArgs a{};
    a.npart = r.npart;
    a.join = join;
    a.count = cnt.get<int64_t>();
    a.u_off = uo.get<int64_t>();
    a.hi_off = ho.get<int64_t>();
    a.lo_off = lo_off.get<int64_t>();
    a.u = reinterpret_cast<double *>(u->dptr);
    a.hi = reinterpret_cast<float *>(hi->dptr);
    a.lo = reinterpret_cast<float *>(lo->dptr);
    launch_split_join(a, r.stream());
  }
};


// Artificial-viscosity stage (av.cu): the plain FP64 stage plus BR1 viscosity eps_e = eps0 sigma_e h_e / N
// from a modal shock sensor.  Op id: rhsStageAV(sensor=none|pp|mlp, eps0=1, c0=0, kappa=1, lo=0.1, hi=0.9);
// the PP switch point is s0 = -(c0 + 4 log10 N).  Roles: u, uNext, resu, Rx..Tz, nx, ny, nz, Fscale, gmap,
// eps, qx, qy, qz (float64 node arrays), matrices Dr, Ds, Dt, LIFT, Fmask, Vinv and, for sensor=mlp, MLP (1 x P
// float32 parameters, read from the device at every launch).  sensorFeatures: the sensor pass alone, writing
// feat (float32, Np per element: unit-norm modal coefficients), sigma (float32 per element: PP activation)
// and, with an MLP role, mlpSigma (the network's output).
struct AvOp : Op {
  int N = 0, mode = 1, ntiles = 0, features = 0;
  int64_t np = 0;
  double eps0 = 1.0, s0 = 0.0, kappa = 1.0;
  float lo = 0.1f, hi = 0.9f;
  Binding *u, *unext = nullptr, *resu = nullptr, *geo[9], *face[4], *gmap, *eps = nullptr, *q[3] = {};
  Binding *mlp = nullptr, *feat = nullptr, *sig = nullptr, *mlps = nullptr;
  DevBuf tiles, dr, ds, dt, vinv, lift, fmask, top, hon, mlp16, qs[3], epsb;
  AvOp(Runner &r, Roles &R, int feats) : features(feats) {
    static const char *gn[9] = {"Rx", "Ry", "Rz", "Sx", "Sy", "Sz", "Tx", "Ty", "Tz"};
    static const char *fn[4] = {"nx", "ny", "nz", "Fscale"};
    const std::string sensor = lower(R.word("sensor", "pp"));
    if (sensor == "none") mode = 0;
    else if (sensor == "pp") mode = 1;
    else if (sensor == "mlp") mode = 2;
    else throw Error(DGK_ERR_INVALID, R.kname + ": sensor must be none, pp or mlp");
    eps0 = R.num("eps0", 1.0);
    kappa = R.num("kappa", 1.0);
    lo = (float)R.num("lo", 0.1);
    hi = (float)R.num("hi", 0.9);
    require(kappa > 0.0 && eps0 >= 0.0, R.kname + ": kappa > 0 and eps0 >= 0");
    u = R.array("u");
    require(u->dev_dtype == DGK_FLOAT64, R.kname + ": the viscosity stage runs in float64");
    for (int i = 0; i < 9; ++i) geo[i] = R.array(gn[i]);
    for (int i = 0; i < 4; ++i) face[i] = R.array(fn[i]);
    gmap = R.array("gmap");
    Binding *Dr = R.matrix("Dr"), *Ds = R.matrix("Ds"), *Dt = R.matrix("Dt"), *L = R.matrix("LIFT"),
            *fm = R.matrix("Fmask"), *Vi = R.matrix("Vinv");
    np = Dr->rows;
    N = order_from_np(np);
    require(N <= 5, R.kname + ": orders 1..5");
    s0 = -(R.num("c0", 0.0) + 4.0 * std::log10((double)N));
    const int nfp = (N + 1) * (N + 2) / 2, nf = 4 * nfp;
    require(u->values_per_elem == np, R.kname + ": u must hold Np values per element");
    for (Binding *b : geo) same_layout(*u, *b, R.kname);
    require(face[0]->values_per_elem == nf && face[0]->dev_dtype == DGK_FLOAT64,
            R.kname + ": face arrays must be float64 with 4*Nfp values per element");
    for (Binding *b : face) same_layout(*face[0], *b, R.kname);
    require(gmap->dev_dtype == DGK_INT32 && gmap->values_per_elem == nf && gmap->offsets == face[0]->offsets,
            R.kname + ": gmap must be int32 with the face arrays' layout");
    require(L->rows == np && L->cols == nf && Vi->rows == np && Vi->cols == np, R.kname + ": LIFT / Vinv shapes");
    if (mode == 2) {
      mlp = R.matrix("MLP");
      require(mlp->rows * mlp->cols == mlp_param_count((int)np) && mlp->dev_dtype == DGK_FLOAT32,
              R.kname + ": MLP must hold " + std::to_string(mlp_param_count((int)np)) + " float32 parameters");
      std::vector<uint16_t> z((size_t)mlp_param_count((int)np) + 8, 0);
      mlp16.upload(z.data(), z.size() * sizeof(uint16_t));
    }
    if (features) {
      feat = R.array("feat");
      sig = R.array("sigma");
      mlps = R.array("mlpSigma", false);
      require(feat->dev_dtype == DGK_FLOAT32 && feat->values_per_elem == np, R.kname + ": feat is float32, Np per element");
      require(sig->dev_dtype == DGK_FLOAT32 && sig->values_per_elem == 1, R.kname + ": sigma is float32, 1 per element");
      if (mlps) same_layout(*sig, *mlps, R.kname);
      // the gradient and viscosity outputs of the sensor pass go to operator-owned scratch
      const size_t nb = sizeof(double) * (size_t)u->offsets.back();
      for (auto &b : qs) b.alloc(nb);
      epsb.alloc(nb);
    } else {
      unext = R.array("uNext");
      resu = R.array("resu");
      eps = R.array("eps");
      q[0] = R.array("qx");
      q[1] = R.array("qy");
      q[2] = R.array("qz");
      for (Binding *b : {unext, resu, eps, q[0], q[1], q[2]}) same_layout(*u, *b, R.kname);
    }
    auto rm = [&](Binding *m, DevBuf &d) { d.upload(m->mat.data(), m->mat.size() * sizeof(double)); };
    rm(Dr, dr);
    rm(Ds, ds);
    rm(Dt, dt);
    rm(Vi, vinv);
    rm(L, lift);
    std::vector<int32_t> fmi(fm->mat.begin(), fm->mat.end());
    for (int32_t v : fmi) require(v >= 0 && v < np, R.kname + ": Fmask entry out of range");
    fmask.upload(fmi.data(), fmi.size() * sizeof(int32_t));
    std::vector<int32_t> tp;
    for (int i = 0; i <= N; ++i)  // modes ordered i, j, k (vandermonde3d.go:15-42)
      for (int j = 0; j <= N - i; ++j)
        for (int k = 0; k <= N - i - j; ++k) tp.push_back(i + j + k == N ? 1 : 0);
    top.upload(tp.data(), tp.size() * sizeof(int32_t));
    // h_e / N with h_e = 2 / max Fscale over the element's face points
    std::vector<double> fs((size_t)face[3]->offsets.back());
    cuda_check(cudaMemcpy(fs.data(), face[3]->dptr, fs.size() * sizeof(double), cudaMemcpyDeviceToHost), "Fscale");
    std::vector<double> h;
    std::vector<AvTile> tl;
    const int te = av_tile_elems(N);
    int64_t eg = 0;
    for (int p = 0; p < r.npart; ++p) {
      for (int64_t e = 0; e < r.K[p]; ++e) {
        double m = 0.0;
        for (int k = 0; k < nf; ++k) m = std::max(m, fs[(size_t)(face[3]->offsets[p] + e * nf + k)]);
        require(m > 0.0, R.kname + ": Fscale must be positive");
        h.push_back(2.0 / m / N);
      }
      for (int64_t s0e = 0; s0e < r.K[p]; s0e += te) {
        AvTile x{};
        x.node_base = u->offsets[p] + s0e * np;
        x.face_base = face[0]->offsets[p] + s0e * nf;
        x.elem_base = eg + s0e;
        x.e1_base = sig ? sig->offsets[p] + s0e : 0;
        x.feat_base = feat ? feat->offsets[p] + s0e * np : 0;
        x.nelem = (int32_t)std::min<int64_t>(te, r.K[p] - s0e);
        x.part = p;
        tl.push_back(x);
      }
      eg += r.K[p];
    }
    hon.upload(h.data(), std::max<size_t>(h.size(), 1) * sizeof(double));
    ntiles = (int)tl.size();
    tiles.upload(tl.data(), std::max<size_t>(tl.size(), 1) * sizeof(AvTile));
  }
  std::vector<std::string> scalar_names() const override {
    if (features) return {};
    return {"a", "b", "dt"};
  }
  void launch(Runner &r, const std::vector<double> &s) override {
    if (ntiles == 0) return;
    AvArgs A{};
    A.tiles = tiles.get<AvTile>();
    A.ntiles = ntiles;
    A.u = reinterpret_cast<const double *>(u->dptr);
    for (int i = 0; i < 9; ++i) A.geo[i] = reinterpret_cast<const double *>(geo[i]->dptr);
    for (int i = 0; i < 4; ++i) A.face[i] = reinterpret_cast<const double *>(face[i]->dptr);
    A.gmap = reinterpret_cast<const int32_t *>(gmap->dptr);
    A.n_u_values = u->offsets.back();
    A.Dr = dr.get<double>();
    A.Ds = ds.get<double>();
    A.Dt = dt.get<double>();
    A.Vinv = vinv.get<double>();
    A.LIFT = lift.get<double>();
    A.fmask = fmask.get<int32_t>();
    A.top = top.get<int32_t>();
    A.h_over_n = hon.get<double>();
    A.mode = mode;
    A.eps0 = eps0;
    A.s0 = s0;
    A.kappa = kappa;
    A.conf_lo = lo;
    A.conf_hi = hi;
    A.status = r.status_word();
    if (mode == 2) {
      launch_to_half(reinterpret_cast<const float *>(mlp->dptr), mlp16.p, mlp_param_count((int)np), r.stream());
      A.mlp16 = mlp16.get<unsigned short>();
    }
    if (features) {
      for (int d = 0; d < 3; ++d) A.q[d] = qs[d].get<double>();
      A.eps = epsb.get<double>();
      A.feat_out = reinterpret_cast<float *>(feat->dptr);
      A.sig_out = reinterpret_cast<float *>(sig->dptr);
      A.mlp_out = mlps ? reinterpret_cast<float *>(mlps->dptr) : nullptr;
      A.prep_only = 1;
      launch_av(N, A, r.num_sms, r.stream());
      return;
    }
    A.u_out = reinterpret_cast<double *>(unext->dptr);
    A.resu = reinterpret_cast<double *>(resu->dptr);
    for (int d = 0; d < 3; ++d) A.q[d] = reinterpret_cast<double *>(q[d]->dptr);
    A.eps = reinterpret_cast<double *>(eps->dptr);
    A.a = s[0];
    A.b = s[1];
    A.dt = s[2];
    launch_av(N, A, r.num_sms, r.stream());
    std::swap(u->dptr, unext->dptr);
  }
};

template <template <typename> class O, typename... A>
std::unique_ptr<Op> typed(int dt, Runner &r, Roles &R, A... a) {
  if (dt == DGK_FLOAT64) return std::make_unique<O<double>>(r, R, a...);
  if (dt == DGK_FLOAT32) return std::make_unique<O<float>>(r, R, a...);
  throw Error(DGK_ERR_UNSUPPORTED, R.kname + ": state arrays must be float64 or float32 on the device");
}

}  // namespace

std::unique_ptr<Op> make_op(Runner &r, KernelConfig &cfg, const std::string &op_id) {
  std::string name;
  std::map<std::string, std::string> kv;
  parse_op(op_id, name, kv);
  Roles R{cfg, kv, cfg.name};
  if (name == "differentiate") return typed<DiffOp>(R.array("U")->dev_dtype, r, R, 0);
  if (name == "computeRHS") return typed<DiffOp>(R.array("u")->dev_dtype, r, R, 1);
  if (name == "updateSolution") return typed<UpdateOp>(R.array("u")->dev_dtype, r, R, 0);
  if (name == "lserkUpdate") return typed<UpdateOp>(R.array("u")->dev_dtype, r, R, 1);
  if (name == "rhsStage") return typed<RhsOp>(R.array("u")->dev_dtype, r, R, 0);
  if (name == "rhsLF") return typed<RhsOp>(R.array("u")->dev_dtype, r, R, 1);
  if (name == "rhsStageMixed") return std::make_unique<MixedOp>(r, R);
  if (name == "rhsStageAV") return std::make_unique<AvOp>(r, R, 0);
  if (name == "sensorFeatures") return std::make_unique<AvOp>(r, R, 1);
  if (name == "splitState") return std::make_unique<SplitJoinOp>(r, R, 0);
  if (name == "joinState") return std::make_unique<SplitJoinOp>(r, R, 1);
  if (name == "matmul") return typed<MatmulOp>(R.array("IN")->dev_dtype, r, R, 0);
  if (name == "matmulAdd") return typed<MatmulOp>(R.array("IN")->dev_dtype, r, R, 1);
  throw Error(DGK_ERR_NOT_FOUND, "unknown operator '" + name + "' (BuildKernel selects a precompiled operator)");
}

}  // namespace dgk
