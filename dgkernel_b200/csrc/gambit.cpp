// Gambit neutral (.neu) mesh reader for tetrahedral meshes (mesh/readers/gambit_reader.go:13-338).
//
// Sections read as the reference does: the control header (NUMNP NELEM NGRPS NBSETS), NODAL COORDINATES
// (vertices in file order; node ids map to those positions), ELEMENTS/CELLS (elements in file order, node ids
// mapped through the node table), ELEMENT GROUP (a group named "p<N>" assigns partition N to its elements;
// EToP exists only when the file has more than one group, unassigned elements stay -1) and BOUNDARY CONDITIONS
// (element/face entries, faces stored 0-based).  Unlike the reference, which skips unsupported element types
// and leaves their connectivity empty, any element that is not a 4-node tetrahedron (type 6) is an error: the
// tet-DG operators are built for tetrahedra only.
#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "mesh.hpp"

namespace dgk {

namespace {

std::string trim(const std::string &s) {
  const size_t a = s.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  const size_t b = s.find_last_not_of(" \t\r\n");
  return s.substr(a, b - a + 1);
}

std::vector<std::string> fields(const std::string &s) {
  std::istringstream is(s);
  std::vector<std::string> out;
  std::string w;
  while (is >> w) out.push_back(w);
  return out;
}

bool to_int(const std::string &s, long long &v) {
  char *end = nullptr;
  v = std::strtoll(s.c_str(), &end, 10);
  return end && *end == '\0' && !s.empty();
}

}  // namespace

GambitMesh read_gambit(const std::string &path) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("cannot open mesh file " + path);
  GambitMesh m;
  std::string line;
  long long numnp = 0, nelem = 0, ngrps = 0, nbsets = 0;
  bool header = false;
  while (std::getline(in, line)) {
    const std::string t = trim(line);
    if (t.find("NUMNP") != std::string::npos && t.find("NELEM") != std::string::npos) {
      if (!std::getline(in, line)) throw std::runtime_error("unexpected end of file after the control header");
      const auto v = fields(line);
      if (v.size() >= 4) {
        to_int(v[0], numnp);
        to_int(v[1], nelem);
        to_int(v[2], ngrps);
        to_int(v[3], nbsets);
      }
      header = true;
      break;
    }
  }
  if (!header) throw std::runtime_error("no control header (NUMNP NELEM ...) in " + path);
  if (numnp < 0 || nelem < 0 || numnp > (1ll << 40) || nelem > (1ll << 40))
    throw std::runtime_error("invalid node or element count in the control header");
  std::map<long long, int64_t> node_index, elem_index;
  while (std::getline(in, line)) {
    const std::string t = trim(line);
    if (t == "ENDOFSECTION") continue;
    if (t.find("NODAL COORDINATES") != std::string::npos) {
      m.VX.assign((size_t)numnp, 0.0);
      m.VY.assign((size_t)numnp, 0.0);
      m.VZ.assign((size_t)numnp, 0.0);
      for (long long i = 0; i < numnp; ++i) {
        if (!std::getline(in, line)) throw std::runtime_error("unexpected end of file reading nodes");
        const auto f = fields(line);
        if (f.size() < 4) throw std::runtime_error("node line " + std::to_string(i + 1) + " has fewer than 4 fields");
        long long id = 0;
        if (!to_int(f[0], id)) throw std::runtime_error("node id is not an integer: " + f[0]);
        m.VX[(size_t)i] = std::strtod(f[1].c_str(), nullptr);
        m.VY[(size_t)i] = std::strtod(f[2].c_str(), nullptr);
        m.VZ[(size_t)i] = std::strtod(f[3].c_str(), nullptr);
        node_index[id] = i;
      }
    } else if (t.find("ELEMENTS/CELLS") != std::string::npos) {
      m.EToV.assign((size_t)(4 * nelem), -1);
      for (long long i = 0; i < nelem; ++i) {
        if (!std::getline(in, line)) throw std::runtime_error("unexpected end of file reading elements");
        const auto f = fields(line);
        long long id = 0, type = 0, nn = 0;
        if (f.size() < 3 || !to_int(f[0], id) || !to_int(f[1], type) || !to_int(f[2], nn))
          throw std::runtime_error("element line " + std::to_string(i + 1) + " is malformed");
        if (type != 6 || nn != 4)
          throw std::runtime_error("element " + std::to_string(id) + " has Gambit type " + std::to_string(type) +
                                   " with " + std::to_string(nn) + " nodes; only 4-node tetrahedra (type 6) are "
                                   "supported");
        if (f.size() < 7) throw std::runtime_error("element " + std::to_string(id) + " lists fewer than 4 nodes");
        for (int c = 0; c < 4; ++c) {
          long long nid = 0;
          auto it = to_int(f[(size_t)(3 + c)], nid) ? node_index.find(nid) : node_index.end();
          if (it == node_index.end())
            throw std::runtime_error("element " + std::to_string(id) + " names unknown node " + f[(size_t)(3 + c)]);
          m.EToV[(size_t)(4 * i + c)] = it->second;
        }
        elem_index[id] = i;
      }
    } else if (t.find("ELEMENT GROUP") != std::string::npos) {
      if (ngrps > 1 && m.EToP.empty()) m.EToP.assign((size_t)nelem, -1);
      if (!std::getline(in, line)) break;
      long long gid = 0, count = 0;
      const auto f = fields(line);
      for (size_t i = 0; i + 1 < f.size(); ++i) {
        if (f[i] == "GROUP:") to_int(f[i + 1], gid);
        if (f[i] == "ELEMENTS:") to_int(f[i + 1], count);
      }
      if (!std::getline(in, line)) break;
      GambitGroup g;
      g.tag = gid;
      g.name = trim(line);
      if (!std::getline(in, line)) break;  // flags line
      long long part = -1, pn = 0;
      if (g.name.size() > 1 && g.name[0] == 'p' && to_int(g.name.substr(1), pn)) part = pn;
      long long got = 0;
      while (got < count && std::getline(in, line)) {
        if (trim(line) == "ENDOFSECTION") break;
        for (const auto &w : fields(line)) {
          long long eid = 0;
          if (!to_int(w, eid) || eid <= 0) continue;
          auto it = elem_index.find(eid);
          if (it != elem_index.end()) {
            g.elements.push_back(it->second);
            if (part >= 0 && !m.EToP.empty()) m.EToP[(size_t)it->second] = part;
          }
          if (++got >= count) break;
        }
      }
      m.groups.push_back(g);
    } else if (t.find("BOUNDARY CONDITIONS") != std::string::npos) {
      for (long long b = 0; b < nbsets; ++b) {
        if (!std::getline(in, line)) break;
        const auto f = fields(line);
        long long itype = 0, nentry = 0, nval = 0;
        if (f.size() < 4) throw std::runtime_error("boundary condition line has fewer than 4 fields");
        if (!to_int(f[1], itype) || !to_int(f[2], nentry) || !to_int(f[3], nval))
          throw std::runtime_error("boundary condition: ITYPE, NENTRY and NVALUES must be integers");
        if (itype != 0 && itype != 1)
          throw std::runtime_error("boundary condition ITYPE " + std::to_string(itype) + " (must be 0 or 1)");
        m.bc_names.push_back(f[0]);
        for (long long i = 0; i < nentry; ++i) {
          if (!std::getline(in, line)) break;
          if (itype != 1) continue;  // node boundary conditions are skipped, as in the reference
          const auto e = fields(line);
          long long eid = 0, et = 0, face = 0;
          if (e.size() < 3 || !to_int(e[0], eid) || !to_int(e[1], et) || !to_int(e[2], face))
            throw std::runtime_error("invalid boundary condition entry");
          auto it = elem_index.find(eid);
          if (it != elem_index.end()) m.bfaces.push_back({it->second, face - 1, (int64_t)b});
        }
      }
    }
  }
  if ((long long)m.VX.size() != numnp) throw std::runtime_error("no NODAL COORDINATES section");
  if ((long long)m.EToV.size() != 4 * nelem) throw std::runtime_error("no ELEMENTS/CELLS section");
  return m;
}

}  // namespace dgk
