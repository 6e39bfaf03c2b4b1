// Host-side mesh setup, see mesh.cpp.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace dgk {

struct FaceConnector {
  int nparts = 0;
  std::vector<int64_t> elems;               // elements per partition
  std::vector<std::vector<int64_t>> pick;   // [src * P + dst] local source nodes
  std::vector<std::vector<int64_t>> place;  // [dst * P + src] local P-buffer positions
};

void kuhn_mesh(int n, int nslab, double lo, double hi, double *VX, double *VY, double *VZ, int64_t *EToV,
               int64_t *EToVp, int64_t *EToP);
void ti_connect3d(int64_t K, const int64_t *EToV, int64_t *EToE, int64_t *EToF);
FaceConnector face_connector(int64_t K, int Nfaces, int Nfp, int Np, const int64_t *vmapP, const int64_t *EToP,
                             int npart);
void face_gather_map(int64_t K, int Nfaces, int Nfp, int Np, const int64_t *vmapP, const int64_t *EToP, int npart,
                     const int64_t *node_off, int32_t *gmap);
// Gather map compressed to one neighbour base per face plus a face-order code (the mixed stage's layout).
// Elements of partition p occupy slots slot_prefix[p] .. slot_prefix[p] + K[p] - 1; each slot holds
// conn[5*slot + f] = value index of the face-f neighbour's first node and conn[5*slot + 4] = the four 8-bit
// codes; table[code*Nfp + i] = node index of face point i within the neighbour.  Throws when a face's points
// do not lie in one element of the state layout, when a base exceeds int32, or past 255 distinct orders.
struct CompactFaces {
  std::vector<int32_t> conn;
  std::vector<uint8_t> table;
  int ncodes = 0;
};
CompactFaces compact_faces(int npart, const int64_t *K, const int64_t *node_off, const int64_t *face_off,
                           const int64_t *slot_prefix, int Np, int Nfp, const int32_t *gmap);
int64_t slot_padded(int64_t k);  // k rounded up to whole 32-element slots

// Tiles of the tensor-core mixed stage with their halos.  Each partition is cut into runs of consecutive
// elements (tiles) of at most max_elems elements, whose first element is a multiple of `align`, and whose
// faces with a neighbour outside the tile number at most max_halo.  Per tile: the halo list (neighbour base,
// face-order code) of those faces, padded to an even entry count; per element slot (slot_prefix layout):
// four words, word f = the face-f neighbour trace's position in the tile's shared-memory slot
// (low 16 bits, in floats from the slot's first value: (neighbour - first element) * Np inside the tile,
// halo_floats + j * Nfp for halo face j) | code << 16, where halo faces carry identity_code (their values
// are stored in this face's point order).  conn is compact_faces' layout.
struct TileHalo {
  std::vector<int32_t> part, nelem;
  std::vector<int64_t> first;      // partition-local first element of each tile
  std::vector<int32_t> halo_off;   // ntiles + 1 entry offsets into halo_list (pairs)
  std::vector<int32_t> halo_list;  // (neighbour base, code) per halo face
  std::vector<uint32_t> tconn;     // 4 words per element slot
};
TileHalo tile_halo(int npart, const int64_t *K, const int64_t *node_off, const int64_t *slot_prefix, int Np, int Nfp,
                   const int32_t *conn, int max_elems, int max_halo, int halo_floats, int identity_code, int align);

// Exchange plan of one rank when partitions are spread over ranks (part_rank[p]), built from the FaceConnector
// pick/place lists (utils/face_connector.go:143-187).  The rank's state array holds its partitions at
// local_off[0..L-1] (value offsets, ascending partition id) and a halo at local_off[L].  For peer rank q the
// wire order is: destination partitions of the receiver ascending, source partitions of the sender ascending,
// pick order within each pair.  gmap covers the rank's face points (packed, partition by partition).
struct HaloPlan {
  std::vector<int32_t> gmap;
  std::vector<int64_t> send_count, recv_count, recv_off;  // per peer rank
  std::vector<int64_t> send_idx;                          // concatenated over peers, local value indices
  int64_t halo_values = 0;
};
HaloPlan halo_plan(int64_t K, int Nfaces, int Nfp, int Np, const int64_t *vmapP, const int64_t *EToP, int npart,
                   const int32_t *part_rank, int nranks, int rank, const int64_t *local_off);

// Gambit neutral file (tetrahedra): vertices in file order, EToV as 0-based vertex positions, EToP from the
// "p<N>" element groups (empty when the file has at most one group), boundary faces (element, 0-based face,
// boundary-set index).
struct GambitGroup {
  int64_t tag = 0;
  std::string name;
  std::vector<int64_t> elements;
};
struct GambitFace {
  int64_t elem, face, set;
};
struct GambitMesh {
  std::vector<double> VX, VY, VZ;
  std::vector<int64_t> EToV, EToP;
  std::vector<GambitGroup> groups;
  std::vector<std::string> bc_names;
  std::vector<GambitFace> bfaces;
};
GambitMesh read_gambit(const std::string &path);

uint64_t splitmix_next(uint64_t &state);
double splitmix_uniform(uint64_t &state);

}  // namespace dgk
