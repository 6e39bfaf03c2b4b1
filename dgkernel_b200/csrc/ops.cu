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
    if (p) cudaFree(p);
    cuda_check(cudaMalloc(&p, std::max<size_t>(bytes, 16)), "cudaMalloc(op buffer)");
    cuda_check(cudaMemcpy(p, h, bytes, cudaMemcpyHostToDevice), "upload op buffer");
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

// Tile list over partitions: up to te consecutive elements of one partition per tile.
std::vector<Tile> make_tiles(const Runner &r, const Binding &node, const Binding *face, int te, int np, int nf) {
  std::vector<Tile> t;
  for (int p = 0; p < r.npart; ++p)
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
  LaunchInfo info;
  RhsOp(Runner &r, Roles &R, int only) : rhs_only(only) {
    static const char *gn[9] = {"Rx", "Ry", "Rz", "Sx", "Sy", "Sz", "Tx", "Ty", "Tz"};
    static const char *fn[4] = {"nx", "ny", "nz", "Fscale"};
    conservative = R.flag("conservative", 0);
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
      auto tl = make_tiles(r, *u, face[0], te_tma, (int)np, nf);
      bool aligned = true;
      for (const Tile &x : tl)
        aligned = aligned && (x.node_base * (int64_t)sizeof(T)) % 16 == 0 &&
                  (x.face_base * (int64_t)sizeof(T)) % 16 == 0 && (x.face_base * 4) % 16 == 0;
      if (aligned) {
        use_tma = true;
        ntiles = (int)tl.size();
        tiles.upload(tl.data(), tl.size() * sizeof(Tile));
      }
    }
    if (!use_tma) {
      auto tl = make_tiles(r, *u, face[0], tile_elems(N), (int)np, nf);
      ntiles = (int)tl.size();
      tiles.upload(tl.data(), tl.size() * sizeof(Tile));
    }
  }
  bool use_tma = false;
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
  if (name == "matmul") return typed<MatmulOp>(R.array("IN")->dev_dtype, r, R, 0);
  if (name == "matmulAdd") return typed<MatmulOp>(R.array("IN")->dev_dtype, r, R, 1);
  throw Error(DGK_ERR_NOT_FOUND, "unknown operator '" + name + "' (BuildKernel selects a precompiled operator)");
}

}  // namespace dgk
