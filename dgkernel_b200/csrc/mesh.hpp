// Host-side mesh setup, see mesh.cpp.
#pragma once
#include <cstdint>
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
uint64_t splitmix_next(uint64_t &state);
double splitmix_uniform(uint64_t &state);

}  // namespace dgk
