// Mesh-side setup on the host: the periodic Kuhn-cube generator, tiConnect3D face matching, the
// FaceConnector pick/place lists and their fused one-address-space gather map.
#include "mesh.hpp"

#include <algorithm>
#include <map>
#include <numeric>
#include <stdexcept>
#include <string>

namespace dgk {

// Corner offsets (x,y,z bits) of the 6 Kuhn tets of a unit cube, all containing the diagonal
// (0,0,0)-(1,1,1), in the order and orientation (J > 0) of utils/mesh_test_helpers.go:353-366.
static const int kKuhn[6][4][3] = {
    {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {1, 1, 1}}, {{0, 0, 0}, {1, 1, 0}, {0, 1, 0}, {1, 1, 1}},
    {{0, 0, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}}, {{0, 0, 0}, {0, 1, 1}, {0, 0, 1}, {1, 1, 1}},
    {{0, 0, 0}, {1, 0, 1}, {1, 0, 0}, {1, 1, 1}}, {{0, 0, 0}, {0, 1, 0}, {0, 1, 1}, {1, 1, 1}}};

void kuhn_mesh(int n, int nslab, double lo, double hi, double *VX, double *VY, double *VZ, int64_t *EToV,
               int64_t *EToVp, int64_t *EToP) {
  if (n < 2) throw std::invalid_argument("Kuhn mesh needs n >= 2");
  if (nslab < 1 || n % nslab) throw std::invalid_argument("n must be a multiple of the slab count");
  const int64_t m = n + 1;
  const double h = (hi - lo) / n;
  for (int64_t i = 0; i < m; ++i)
    for (int64_t j = 0; j < m; ++j)
      for (int64_t k = 0; k < m; ++k) {
        const int64_t v = (i * m + j) * m + k;
        VX[v] = lo + h * (double)i;
        VY[v] = lo + h * (double)j;
        VZ[v] = lo + h * (double)k;
      }
  const int per = n / nslab;
  for (int64_t i = 0; i < n; ++i)
    for (int64_t j = 0; j < n; ++j)
      for (int64_t k = 0; k < n; ++k) {
        const int64_t cube = (i * n + j) * n + k;
        for (int t = 0; t < 6; ++t) {
          const int64_t e = cube * 6 + t;
          for (int c = 0; c < 4; ++c) {
            const int64_t gi = i + kKuhn[t][c][0], gj = j + kKuhn[t][c][1], gk = k + kKuhn[t][c][2];
            EToV[e * 4 + c] = (gi * m + gj) * m + gk;
            EToVp[e * 4 + c] = ((gi % n) * n + (gj % n)) * n + (gk % n);
          }
          EToP[e] = i / per;
        }
      }
}

// Faces {0,1,2}, {0,1,3}, {1,2,3}, {0,2,3} keyed by their sorted vertex triple
// (element/library/gonudg/ticonnect3d.go:24-102).  Equal keys are linked pairwise in sorted order.
void ti_connect3d(int64_t K, const int64_t *EToV, int64_t *EToE, int64_t *EToF) {
  static const int fv[4][3] = {{0, 1, 2}, {0, 1, 3}, {1, 2, 3}, {0, 2, 3}};
  int64_t nn = 0;
  for (int64_t i = 0; i < 4 * K; ++i) nn = std::max(nn, EToV[i] + 1);
  struct Key {
    int64_t id, slot;
  };
  std::vector<Key> keys((size_t)(4 * K));
  for (int64_t e = 0; e < K; ++e)
    for (int f = 0; f < 4; ++f) {
      int64_t v[3] = {EToV[e * 4 + fv[f][0]], EToV[e * 4 + fv[f][1]], EToV[e * 4 + fv[f][2]]};
      std::sort(v, v + 3);
      keys[(size_t)(e * 4 + f)] = {(v[0] * nn + v[1]) * nn + v[2], e * 4 + f};
    }
  std::sort(keys.begin(), keys.end(), [](const Key &a, const Key &b) {
    return a.id != b.id ? a.id < b.id : a.slot < b.slot;
  });
  for (int64_t e = 0; e < K; ++e)
    for (int f = 0; f < 4; ++f) {
      EToE[e * 4 + f] = e;
      EToF[e * 4 + f] = f;
    }
  for (size_t i = 0; i + 1 < keys.size(); ++i) {
    if (keys[i].id != keys[i + 1].id) continue;
    const int64_t a = keys[i].slot, b = keys[i + 1].slot;
    EToE[a] = b / 4;
    EToF[a] = b % 4;
    EToE[b] = a / 4;
    EToF[b] = a % 4;
  }
}

// NewFaceConnector + BuildIndices + Verify (utils/face_connector.go:43-253).  Local element numbers
// follow increasing global id inside each partition.
FaceConnector face_connector(int64_t K, int Nfaces, int Nfp, int Np, const int64_t *vmapP, const int64_t *EToP,
                             int npart) {
  if (K <= 0 || Nfaces <= 0 || Nfp <= 0 || Np <= 0) throw std::invalid_argument("invalid dimensions");
  int P = 0;
  for (int64_t e = 0; e < K; ++e) {
    if (EToP[e] < 0) throw std::invalid_argument("negative partition id");
    P = std::max<int>(P, (int)EToP[e] + 1);
  }
  if (npart > 0 && P != npart) throw std::invalid_argument("EToP partition count does not match npart");
  FaceConnector fc;
  fc.nparts = P;
  fc.elems.assign(P, 0);
  std::vector<int64_t> local((size_t)K);
  for (int64_t e = 0; e < K; ++e) local[(size_t)e] = fc.elems[(size_t)EToP[e]]++;
  fc.pick.assign((size_t)P * P, {});
  fc.place.assign((size_t)P * P, {});
  const int64_t NF = (int64_t)Nfaces * Nfp;
  for (int p = 0; p < P; ++p)  // partition p in ascending global element order
    for (int64_t ge = 0; ge < K; ++ge) {
      if (EToP[ge] != p) continue;
      const int64_t le = local[(size_t)ge];
      for (int64_t q = 0; q < NF; ++q) {
        const int64_t src = vmapP[ge * NF + q];
        if (src < 0 || src >= K * Np) throw std::invalid_argument("vmapP entry out of range");
        const int64_t se = src / Np;
        const int sp = (int)EToP[se];
        fc.pick[(size_t)sp * P + p].push_back(local[(size_t)se] * Np + src % Np);
        fc.place[(size_t)p * P + sp].push_back(le * NF + q);
      }
    }
  // Verify: index validity, pick/place correspondence, conservation
  int64_t total = 0;
  for (int p = 0; p < P; ++p)
    for (int q = 0; q < P; ++q) {
      for (int64_t v : fc.pick[(size_t)p * P + q])
        if (v < 0 || v >= fc.elems[p] * Np)
          throw std::runtime_error("invalid pick index for partition " + std::to_string(p));
      if (fc.pick[(size_t)p * P + q].size() != fc.place[(size_t)q * P + p].size())
        throw std::runtime_error("pick/place length mismatch");
      total += (int64_t)fc.pick[(size_t)p * P + q].size();
    }
  if (total != K * NF) throw std::runtime_error("conservation error: picks != face points");
  return fc;
}

void face_gather_map(int64_t K, int Nfaces, int Nfp, int Np, const int64_t *vmapP, const int64_t *EToP, int npart,
                     const int64_t *node_off, int32_t *gmap) {
  FaceConnector fc = face_connector(K, Nfaces, Nfp, Np, vmapP, EToP, npart);
  const int P = fc.nparts;
  const int64_t NF = (int64_t)Nfaces * Nfp;
  std::vector<int64_t> face_base(P + 1, 0);  // P-buffers of all partitions back to back
  for (int p = 0; p < P; ++p) face_base[p + 1] = face_base[p] + fc.elems[p] * NF;
  for (int dst = 0; dst < P; ++dst)
    for (int src = 0; src < P; ++src) {
      const auto &pk = fc.pick[(size_t)src * P + dst];
      const auto &pl = fc.place[(size_t)dst * P + src];
      for (size_t i = 0; i < pk.size(); ++i) {
        const int64_t v = node_off[src] + pk[i];
        if (v > INT32_MAX) throw std::runtime_error("gather index exceeds int32");
        gmap[face_base[dst] + pl[i]] = (int32_t)v;
      }
    }
}

HaloPlan halo_plan(int64_t K, int Nfaces, int Nfp, int Np, const int64_t *vmapP, const int64_t *EToP, int npart,
                   const int32_t *part_rank, int nranks, int rank, const int64_t *local_off) {
  if (nranks < 1 || rank < 0 || rank >= nranks) throw std::invalid_argument("rank outside 0..nranks-1");
  for (int p = 0; p < npart; ++p)
    if (part_rank[p] < 0 || part_rank[p] >= nranks) throw std::invalid_argument("partition assigned to no rank");
  FaceConnector fc = face_connector(K, Nfaces, Nfp, Np, vmapP, EToP, npart);
  const int P = fc.nparts;
  const int64_t NF = (int64_t)Nfaces * Nfp;
  std::vector<int> local;  // this rank's partitions, ascending
  std::vector<int> lidx((size_t)P, -1);
  for (int p = 0; p < P; ++p)
    if (part_rank[p] == rank) {
      lidx[(size_t)p] = (int)local.size();
      local.push_back(p);
    }
  const int L = (int)local.size();
  std::vector<int64_t> face_base((size_t)L + 1, 0);  // the rank's P-buffers back to back
  for (int i = 0; i < L; ++i) face_base[(size_t)i + 1] = face_base[(size_t)i] + fc.elems[(size_t)local[(size_t)i]] * NF;
  HaloPlan hp;
  hp.gmap.assign((size_t)face_base[(size_t)L], -1);
  hp.send_count.assign((size_t)nranks, 0);
  hp.recv_count.assign((size_t)nranks, 0);
  hp.recv_off.assign((size_t)nranks, 0);
  auto put = [&](int64_t pos, int64_t v) {
    if (v > INT32_MAX) throw std::runtime_error("gather index exceeds int32");
    hp.gmap[(size_t)pos] = (int32_t)v;
  };
  // neighbours in this rank's own partitions
  for (int i = 0; i < L; ++i) {
    const int dst = local[(size_t)i];
    for (int src = 0; src < P; ++src) {
      if (part_rank[src] != rank) continue;
      const auto &pk = fc.pick[(size_t)src * P + dst];
      const auto &pl = fc.place[(size_t)dst * P + src];
      for (size_t k = 0; k < pk.size(); ++k) put(face_base[(size_t)i] + pl[k], local_off[lidx[(size_t)src]] + pk[k]);
    }
  }
  // received from peer q, in wire order, into the halo
  int64_t h = 0;
  for (int q = 0; q < nranks; ++q) {
    hp.recv_off[(size_t)q] = h;
    if (q == rank) continue;
    for (int i = 0; i < L; ++i) {
      const int dst = local[(size_t)i];
      for (int src = 0; src < P; ++src) {
        if (part_rank[src] != q) continue;
        const auto &pl = fc.place[(size_t)dst * P + src];
        for (size_t k = 0; k < pl.size(); ++k) put(face_base[(size_t)i] + pl[k], local_off[L] + h++);
      }
    }
    hp.recv_count[(size_t)q] = h - hp.recv_off[(size_t)q];
  }
  hp.halo_values = h;
  // sent to peer q, in the order q receives them
  for (int q = 0; q < nranks; ++q) {
    if (q == rank) continue;
    const int64_t before = (int64_t)hp.send_idx.size();
    for (int dst = 0; dst < P; ++dst) {
      if (part_rank[dst] != q) continue;
      for (int i = 0; i < L; ++i) {
        const int src = local[(size_t)i];
        for (int64_t v : fc.pick[(size_t)src * P + dst]) hp.send_idx.push_back(local_off[(size_t)i] + v);
      }
    }
    hp.send_count[(size_t)q] = (int64_t)hp.send_idx.size() - before;
  }
  for (int32_t g : hp.gmap)
    if (g < 0) throw std::runtime_error("halo plan: a face point has no source");
  return hp;
}

int64_t slot_padded(int64_t k) { return (k + 31) / 32 * 32; }

CompactFaces compact_faces(int npart, const int64_t *K, const int64_t *node_off, const int64_t *face_off,
                           const int64_t *slot_prefix, int Np, int Nfp, const int32_t *gmap) {
  if (Np > 255) throw std::runtime_error("compact faces: Np above 255 does not fit the 8-bit table");
  CompactFaces out;
  out.conn.assign((size_t)(slot_prefix[npart] * 5), 0);
  std::map<std::vector<uint8_t>, int> codes;
  std::vector<uint8_t> order((size_t)Nfp);
  const int64_t NF = 4 * (int64_t)Nfp;
  for (int p = 0; p < npart; ++p)
    for (int64_t e = 0; e < K[p]; ++e) {
      uint32_t packed = 0;
      for (int f = 0; f < 4; ++f) {
        const int32_t *g = gmap + face_off[p] + e * NF + (int64_t)f * Nfp;
        // partition holding the first face point, then the element base within it
        const int q = (int)(std::upper_bound(node_off, node_off + npart, (int64_t)g[0]) - node_off) - 1;
        if (q < 0 || g[0] >= node_off[q] + K[q] * Np) throw std::runtime_error("compact faces: gather index outside every partition of the state");
        const int64_t base = node_off[q] + (g[0] - node_off[q]) / Np * Np;
        if (base > INT32_MAX) throw std::runtime_error("compact faces: neighbour base exceeds int32");
        for (int i = 0; i < Nfp; ++i) {
          const int64_t j = (int64_t)g[i] - base;
          if (j < 0 || j >= Np) throw std::runtime_error("compact faces: the points of one face span two elements");
          order[(size_t)i] = (uint8_t)j;
        }
        auto it = codes.find(order);
        int code;
        if (it == codes.end()) {
          code = (int)codes.size();
          if (code > 254) throw std::runtime_error("compact faces: more than 255 distinct face orders");
          codes.emplace(order, code);
          out.table.insert(out.table.end(), order.begin(), order.end());
        } else {
          code = it->second;
        }
        out.conn[(size_t)((slot_prefix[p] + e) * 5 + f)] = (int32_t)base;
        packed |= (uint32_t)code << (8 * f);
      }
      out.conn[(size_t)((slot_prefix[p] + e) * 5 + 4)] = (int32_t)packed;
    }
  out.ncodes = (int)codes.size();
  return out;
}

TileHalo tile_halo(int npart, const int64_t *K, const int64_t *node_off, const int64_t *slot_prefix, int Np, int Nfp,
                   const int32_t *conn, int max_elems, int max_halo, int halo_floats, int identity_code, int align) {
  if (align < 1 || max_elems < align || max_halo < 4 * align || (max_halo & 1))
    throw std::runtime_error("tile halo: limits must satisfy max_elems >= align, max_halo >= 4 align, max_halo even");
  if ((int64_t)max_elems * Np > halo_floats || (int64_t)halo_floats + (int64_t)max_halo * Nfp > 65536)
    throw std::runtime_error("tile halo: slot positions do not fit 16 bits");
  if (identity_code < 0 || identity_code > 255) throw std::runtime_error("tile halo: identity code outside 8 bits");
  TileHalo out;
  out.tconn.assign((size_t)(slot_prefix[npart] * 4), 0u);
  out.halo_off.push_back(0);
  for (int p = 0; p < npart; ++p) {
    const int64_t lo = node_off[p], hi = node_off[p] + K[p] * Np;
    // partition-local element of the face-f neighbour of element e; -1 outside this partition
    auto nbr = [&](int64_t e, int f) -> int64_t {
      const int64_t nb = conn[(size_t)((slot_prefix[p] + e) * 5 + f)];
      return (nb >= lo && nb < hi) ? (nb - lo) / Np : -1;
    };
    for (int64_t s0 = 0; s0 < K[p];) {
      // grow the tile one element at a time, keeping the count of faces whose neighbour lies outside it; the
      // tile is the longest prefix that ends on an aligned boundary (or the partition's end) within max_halo
      const int64_t mmax = std::min<int64_t>(max_elems, K[p] - s0);
      int64_t best = 0;
      int64_t c = 0;
      for (int64_t m = 1; m <= mmax; ++m) {
        const int64_t x = s0 + m - 1;
        int64_t seen[4];
        int ns = 0;
        for (int f = 0; f < 4; ++f) {
          const int64_t y = nbr(x, f);
          if (y < s0 || y > x) {
            ++c;  // neighbour outside the tile so far
            continue;
          }
          if (y == x) continue;  // a face whose neighbour is the element itself
          bool dup = false;
          for (int i = 0; i < ns; ++i) dup |= seen[i] == y;
          if (dup) continue;
          seen[ns++] = y;
          for (int g = 0; g < 4; ++g) c -= nbr(y, g) == x;  // y's faces towards x are inside now
        }
        if (c <= max_halo && (m % align == 0 || s0 + m == K[p])) best = m;
      }
      if (best == 0) throw std::runtime_error("tile halo: an aligned group of elements exceeds the halo capacity");
      int32_t j = 0;
      for (int64_t e = s0; e < s0 + best; ++e) {
        const int64_t sl = slot_prefix[p] + e;
        const uint32_t codes = (uint32_t)conn[(size_t)(sl * 5 + 4)];
        for (int f = 0; f < 4; ++f) {
          const int64_t y = nbr(e, f);
          const uint32_t code = (codes >> (8 * f)) & 0xffu;
          uint32_t word;
          if (y >= s0 && y < s0 + best) {
            word = (uint32_t)((y - s0) * Np) | (code << 16);
          } else {
            out.halo_list.push_back(conn[(size_t)(sl * 5 + f)]);
            out.halo_list.push_back((int32_t)code);
            word = (uint32_t)(halo_floats + j * Nfp) | ((uint32_t)identity_code << 16);
            ++j;
          }
          out.tconn[(size_t)(sl * 4 + f)] = word;
        }
      }
      if (j & 1) {  // even entry count (16-byte copies): repeat the last entry
        const size_t n = out.halo_list.size();
        out.halo_list.push_back(out.halo_list[n - 2]);
        out.halo_list.push_back(out.halo_list[n - 1]);
      }
      if (out.halo_list.size() / 2 > (size_t)INT32_MAX) throw std::runtime_error("tile halo: more than 2^31 entries");
      out.halo_off.push_back((int32_t)(out.halo_list.size() / 2));
      out.part.push_back(p);
      out.first.push_back(s0);
      out.nelem.push_back((int32_t)best);
      s0 += best;
    }
  }
  return out;
}

uint64_t splitmix_next(uint64_t &state) {
  state += 0x9E3779B97F4A7C15ull;
  uint64_t z = state;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

double splitmix_uniform(uint64_t &state) { return (double)(splitmix_next(state) >> 11) * (1.0 / 9007199254740992.0); }

}  // namespace dgk
