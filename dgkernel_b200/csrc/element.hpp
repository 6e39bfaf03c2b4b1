// Host-side reference tetrahedron (FP64), see element.cpp.
#pragma once
#include <vector>

namespace dgk {

struct RefElement {
  explicit RefElement(int order);
  int N, Np, Nfp;
  std::vector<double> r, s, t;                       // reference nodes (Np)
  std::vector<double> V, Vinv, MassMatrix, M, Minv;  // Np x Np, row-major
  std::vector<double> Dr, Ds, Dt;                    // Np x Np, row-major
  std::vector<double> LIFT;                          // Np x 4Nfp, row-major
  std::vector<int> Fmask;                            // 4 x Nfp
};

std::vector<double> invert(const std::vector<double> &M, int n);
std::vector<double> matmul(const std::vector<double> &A, const std::vector<double> &B, int m, int k, int n);
std::vector<double> transpose(const std::vector<double> &A, int m, int n);

}  // namespace dgk
