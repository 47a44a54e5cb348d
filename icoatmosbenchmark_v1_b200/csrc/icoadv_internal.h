// Internal declarations shared by the host library and the CUDA kernels.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "icoadv.h"

namespace icoadv {

constexpr int kVlink = 5;   // ADM_vlink: regions around a pole
constexpr int kGallPl = 6;  // ADM_gall_pl
constexpr int kLallPl = 2;  // ADM_lall_pl

struct Link {
  int rgn, dir;
};
struct Copy {
  int dst, src;  // point indices
};

// Region management and the composed halo fill of one whole grid.
struct Topology {
  int glevel, rlevel, nrgn, nmax, gall_1d, gall, gmin, gmax;
  std::vector<Link> edge;      // [rgn][4] neighbour across SW, NW, NE, SE
  std::vector<int> vert_num;   // [rgn][4] regions around corners W, N, E, S
  std::vector<Link> vert_tab;  // [rgn][4][kVlink]
  int rgn4pl[2];               // first region whose N (S) corner is the pole
  int pole_ring[2][kVlink];    // regions around each pole, walkaround order
  std::vector<int> have_sgp;   // [rgn] region holds a pentagon at (gmin,gmin)

  Topology(int glevel, int rlevel);
  Link link(int r, int e) const { return edge[(r - 1) * 4 + (e - 1)]; }
  int vnum(int r, int v) const { return vert_num[(r - 1) * 4 + (v - 1)]; }
  Link vtab(int r, int v, int n) const { return vert_tab[((r - 1) * 4 + (v - 1)) * kVlink + (n - 1)]; }
  int npoints() const { return nrgn * gall + kLallPl * kGallPl; }
  int pt(int r, int i, int j) const;
  int ptp(int p, int v) const;
  std::vector<Copy> copy_sequence(bool pole_fill) const;
  int build_plan(bool pole_fill, std::vector<int> &dst, std::vector<int> &src) const;
};

void set_error(const std::string &msg);

}  // namespace icoadv
