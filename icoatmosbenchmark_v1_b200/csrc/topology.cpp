// Region topology and the single-GPU halo/pole fill plan.
//
// The reference fills halos with COMM_data_transfer
// (kernels/NICAM/communication/src/mod_comm.f90:1506-1891): per process a
// list of copies p2r, r2p, r2r, then "singular" halo-to-halo copies that
// read halo cells the r2r copies just wrote (mod_comm.f90:1868-1884), and,
// for COMM_var (mod_comm.f90:1895-2101), a halo -> pole-centre copy first.
// On one GPU every region is local, so the whole sequence collapses to one
// gather dst[p] = src[s(p)] over "points" (region cells and pole cells).
// This file replays the reference's list construction on the host, composes
// the sequence (a later copy that reads a cell an earlier copy wrote reads
// that copy's source instead), drops self-copies, and checks that no source
// is also a destination, so one parallel in-place gather is exact.
//
// Topology tables follow RGNMNG_generate_ico / RGNMNG_vertex_walkaround
// (mod_adm.f90:629-894); the diamond adjacency table must be the reference's.
#include "icoadv_internal.h"

#include <algorithm>
#include <cstring>
#include <vector>

namespace icoadv {

namespace {
enum Edge { SW = 1, NW = 2, NE = 3, SE = 4 };
enum Vert { W = 1, N = 2, E = 3, S = 4 };
}  // namespace

// Diamond adjacency (SW, NW, NE, SE neighbours of diamond 1..10), the
// icosahedral default topology of the reference (mod_adm.f90:662-671).
static const int kDiamondNeighbour[10][4] = {
    {6, 5, 2, 10}, {10, 1, 3, 9}, {9, 2, 4, 8}, {8, 3, 5, 7}, {7, 4, 1, 6},
    {7, 5, 1, 10}, {8, 4, 5, 6}, {9, 3, 4, 7}, {10, 2, 3, 8}, {6, 1, 2, 9}};

Topology::Topology(int glevel_, int rlevel_) : glevel(glevel_), rlevel(rlevel_) {
  const int rl1 = 1 << rlevel, rl2 = rl1 * rl1;
  nrgn = 10 * rl2;
  nmax = 1 << (glevel - rlevel);
  gall_1d = nmax + 2;
  gall = gall_1d * gall_1d;
  gmin = 2;
  gmax = nmax + 1;
  edge.assign(nrgn * 4, {0, 0});
  auto id = [&](int d, int i, int j) { return (d - 1) * rl2 + (j - 1) * rl1 + i; };
  for (int d = 1; d <= 10; ++d) {
    const bool north = d <= 5;
    const int *nb = kDiamondNeighbour[d - 1];
    for (int i = 1; i <= rl1; ++i)
      for (int j = 1; j <= rl1; ++j) {
        const int r = id(d, i, j);
        Link *e = &edge[(r - 1) * 4];
        // south-west edge
        if (j > 1) e[SW - 1] = {id(d, i, j - 1), NE};
        else if (north) e[SW - 1] = {id(nb[0], i, rl1), NE};
        else e[SW - 1] = {id(nb[0], rl1, rl1 + 1 - i), SE};
        // north-west edge
        if (i > 1) e[NW - 1] = {id(d, i - 1, j), SE};
        else if (north) e[NW - 1] = {id(nb[1], rl1 + 1 - j, rl1), NE};
        else e[NW - 1] = {id(nb[1], rl1, j), SE};
        // north-east edge
        if (j < rl1) e[NE - 1] = {id(d, i, j + 1), SW};
        else if (north) e[NE - 1] = {id(nb[2], 1, rl1 + 1 - i), NW};
        else e[NE - 1] = {id(nb[2], i, 1), SW};
        // south-east edge
        if (i < rl1) e[SE - 1] = {id(d, i + 1, j), NW};
        else if (north) e[SE - 1] = {id(nb[3], 1, j), NW};
        else e[SE - 1] = {id(nb[3], rl1 + 1 - j, 1), SW};
      }
  }
  // walk around each region corner; a corner shared by k regions closes after k hops
  vert_num.assign(nrgn * 4, 0);
  vert_tab.assign(nrgn * 4 * kVlink, {-1, -1});
  for (int r = 1; r <= nrgn; ++r)
    for (int v = W; v <= S; ++v) {
      int rg = r, dir = v;  // corner W starts along edge SW, N along NW, ...
      int hops = 0;
      do {
        if (hops < kVlink) vert_tab[((r - 1) * 4 + (v - 1)) * kVlink + hops] = {rg, dir};
        const Link nx = edge[(rg - 1) * 4 + (dir - 1)];
        rg = nx.rgn;
        dir = nx.dir == 1 ? 4 : nx.dir - 1;
        ++hops;
      } while (rg != r && hops < 64);
      vert_num[(r - 1) * 4 + (v - 1)] = hops;
    }
  rgn4pl[0] = rgn4pl[1] = -1;
  for (int p = 0; p < 2; ++p) {
    const int corner = p == 0 ? N : S;
    for (int r = 1; r <= nrgn && rgn4pl[p] < 0; ++r)
      if (vnum(r, corner) == kVlink) rgn4pl[p] = r;
    for (int v = 0; v < kVlink; ++v) pole_ring[p][v] = vtab(rgn4pl[p], corner, v + 1).rgn;
  }
  have_sgp.resize(nrgn);
  for (int r = 1; r <= nrgn; ++r) have_sgp[r - 1] = vnum(r, W) == 3 ? 1 : 0;
}

// point index of region cell (i,j) (1-based) of region r (1-based); pole v of pole p
int Topology::pt(int r, int i, int j) const { return (r - 1) * gall + (j - 1) * gall_1d + (i - 1); }
int Topology::ptp(int p, int v) const { return nrgn * gall + p * kGallPl + (v - 1); }

std::vector<Copy> Topology::copy_sequence(bool pole_fill) const {
  std::vector<Copy> p2r, r2p, r2r, sing, pre;
  const int g0 = gmin, g1 = gmax, n = g1 - g0 + 1;
  for (int r = 1; r <= nrgn; ++r) {
    auto add = [&](int i, int j, int rr, int ir, int jr) { r2r.push_back({pt(r, i, j), pt(rr, ir, jr)}); };
    const Link sw = link(r, SW), nw = link(r, NW), ne = link(r, NE), se = link(r, SE);
    for (int m = 1; m <= n; ++m) {  // edge strips (mod_comm.f90:256-438)
      if (sw.dir == NE) add(g0 - 1 + m, g0 - 1, sw.rgn, g0 - 1 + m, g1);
      if (sw.dir == SE) add(g0 - 1 + m, g0 - 1, sw.rgn, g1, g1 + 1 - m);
      if (nw.dir == SE) add(g0 - 1, g0 - 1 + m, nw.rgn, g1, g0 - 1 + m);
      if (nw.dir == NE) add(g0 - 1, g0 - 1 + m, nw.rgn, g1 + 1 - m, g1);
      if (ne.dir == SW) add(g0 - 1 + m, g1 + 1, ne.rgn, g0 - 1 + m, g0);
      if (ne.dir == NW) add(g0 + m, g1 + 1, ne.rgn, g0, g1 + 1 - m);
      if (se.dir == NW) add(g1 + 1, g0 - 1 + m, se.rgn, g0, g0 - 1 + m);
      if (se.dir == SW) add(g1 + 1, g0 + m, se.rgn, g1 + 1 - m, g0);
    }
    // corners shared by four regions (mod_comm.f90:440-591)
    auto far_corner = [&](int dirv, int &ir, int &jr) {
      ir = -1, jr = -1;
      if (dirv == N) ir = g0, jr = g1;
      else if (dirv == E) ir = g1, jr = g1;
      else if (dirv == S) ir = g1, jr = g0;
    };
    if (vnum(r, W) == 4) {
      const Link x = vtab(r, W, 3);
      int ir, jr;
      far_corner(x.dir, ir, jr);
      add(g0 - 1, g0 - 1, x.rgn, ir, jr);
    }
    if (vnum(r, N) == 4) {
      const Link x = vtab(r, N, 3);
      int ir, jr;
      if (x.dir == W) { add(g0, g1 + 1, x.rgn, g0, g0); ir = g0; jr = g0 + 1; }
      else far_corner(x.dir, ir, jr);
      add(g0 - 1, g1 + 1, x.rgn, ir, jr);
    }
    if (vnum(r, E) == 4 && vtab(r, E, 3).dir == W) add(g1 + 1, g1 + 1, vtab(r, E, 3).rgn, g0, g0);
    if (vnum(r, S) == 4) {
      const Link x = vtab(r, S, 3);
      int ir, jr;
      if (x.dir == W) { add(g1 + 1, g0, x.rgn, g0, g0); ir = g0 + 1; jr = g0; }
      else far_corner(x.dir, ir, jr);
      add(g1 + 1, g0 - 1, x.rgn, ir, jr);
    }
    // singular halo-to-halo copies (mod_comm.f90:1414-1462)
    if (vnum(r, W) == 3) sing.push_back({pt(r, g0 - 1, g0 - 1), pt(r, g0, g0 - 1)});
    if (vnum(r, N) != 4) sing.push_back({pt(r, g0 - 1, g1 + 1), pt(r, g0 - 1, g1)});
    if (vnum(r, S) != 4) sing.push_back({pt(r, g1 + 1, g0 - 1), pt(r, g1 + 1, g0)});
  }
  // pole <-> region (mod_comm.f90:1000-1188); ring slot of ring position v is v, 1 -> 6
  for (int p = 0; p < 2; ++p) {
    const int corner = p == 0 ? N : S;
    for (int v = 1; v <= kVlink; ++v) {
      const int r = pole_ring[p][v - 1];
      if (vnum(r, corner) != kVlink) continue;
      const int slot = v < 2 ? kGallPl : v;
      const int hi = p == 0 ? g0 : g1 + 1, hj = p == 0 ? g1 + 1 : g0;  // region halo next to the pole
      const int ii = p == 0 ? g0 : g1, ij = p == 0 ? g1 : g0;          // region cell next to the pole
      p2r.push_back({pt(r, hi, hj), ptp(p, 1)});
      r2p.push_back({ptp(p, slot), pt(r, ii, ij)});
    }
    if (pole_fill) {  // COMM_var: pole centre <- halo of rgn4pl, before the transfer
      const int r = rgn4pl[p];
      const int hi = p == 0 ? g0 : g1 + 1, hj = p == 0 ? g1 + 1 : g0;
      pre.push_back({ptp(p, 1), pt(r, hi, hj)});
    }
  }
  std::vector<Copy> seq;
  for (auto *v : {&pre, &p2r, &r2p, &r2r, &sing}) seq.insert(seq.end(), v->begin(), v->end());
  return seq;
}

int Topology::build_plan(bool pole_fill, std::vector<int> &dst, std::vector<int> &src) const {
  const int np = npoints();
  std::vector<int> from(np);
  for (int p = 0; p < np; ++p) from[p] = p;
  for (const Copy &c : copy_sequence(pole_fill)) from[c.dst] = from[c.src];
  dst.clear();
  src.clear();
  std::vector<char> is_dst(np, 0);
  for (int p = 0; p < np; ++p)
    if (from[p] != p) {
      dst.push_back(p);
      src.push_back(from[p]);
      is_dst[p] = 1;
    }
  for (int s : src)
    if (is_dst[s]) return ICA_ERR_INTERNAL;  // would need a two-phase gather
  return ICA_OK;
}

}  // namespace icoadv

using icoadv::Topology;

extern "C" int ica_comm_plan(int glevel, int rlevel, int pole_fill, int *n, int *dst, int *src) {
  if (glevel < 1 || rlevel < 0 || rlevel > glevel || glevel > 12 || !n) return ICA_ERR_ARG;
  Topology t(glevel, rlevel);
  std::vector<int> d, s;
  int rc = t.build_plan(pole_fill != 0, d, s);
  if (rc) return rc;
  if (dst && src) {
    if (*n < (int)d.size()) return ICA_ERR_ARG;
    std::memcpy(dst, d.data(), sizeof(int) * d.size());
    std::memcpy(src, s.data(), sizeof(int) * s.size());
  }
  *n = (int)d.size();
  return ICA_OK;
}

extern "C" int ica_topology_info(int glevel, int rlevel, int *have_sgp, int *rgn4pl, int *pole_ring) {
  if (glevel < 1 || rlevel < 0 || rlevel > glevel || glevel > 12) return ICA_ERR_ARG;
  Topology t(glevel, rlevel);
  if (have_sgp) std::memcpy(have_sgp, t.have_sgp.data(), sizeof(int) * t.nrgn);
  if (rgn4pl) rgn4pl[0] = t.rgn4pl[0], rgn4pl[1] = t.rgn4pl[1];
  if (pole_ring)
    for (int p = 0; p < 2; ++p)
      for (int v = 0; v < icoadv::kVlink; ++v) pole_ring[p * icoadv::kVlink + v] = t.pole_ring[p][v];
  return ICA_OK;
}
