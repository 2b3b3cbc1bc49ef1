// Host-side FP64 setup tables of the MLFMA operator (the work of the
// reference's setup_mlfma.cpp:50-695 and integrate.cpp), built without any GPU.
//
// Tables that do not depend on cluster numbering (near-field blocks, P2M/L2P
// plane-wave coefficients, Lagrange interpolators and their transposes, shift
// phases, translation operators, receiver interpolators) are stored in the
// reference's own layouts so that they can be compared entry by entry with the
// oracle.  Cluster numbering is the library's own: clusters of level i form an
// n_i x n_i raster (row 0 at the top), so near and far lists become stencils and
// are not stored.
#pragma once

#include <complex>
#include <string>
#include <vector>

namespace isg {

using cd = std::complex<double>;

struct HostTables {
  // geometry (mom.cpp:4-6,136-138)
  int L = 0;          // levels; level 0 is the root, level L-1 the leaves
  int box = 8, bb = 64;
  int side = 0;       // pixels per side = box * 2^(L-1)
  int nleaf = 0;      // leaves per side
  int U = 0;          // unknowns
  int ninter = 30, beta = 5, numrx = 0;
  double k0 = 0, res = 0.1;
  std::vector<int> nclus, nsamp, nterm;  // per level
  std::vector<double> csize;             // cluster side per level

  // leaf stage tables (setup_mlfma.cpp:492-505, 544-553)
  std::vector<cd> near;   // [9 slots][bb testing][bb basis]; slot = (row offset+1)*3 + (col offset+1)
  std::vector<cd> coeff;  // [ns_leaf][bb]   P2M plane-wave coefficients (with res^2)
  std::vector<cd> basis;  // [bb][ns_leaf]   L2P plane-wave basis (with i/4/ns)

  // per-level tables
  std::vector<std::vector<double>> interp;  // level i < L-1: [ns_i][ninter]
  std::vector<std::vector<int>> intind;     // level i < L-1: [ns_i][ninter] indices into level i+1
  std::vector<std::vector<double>> anterp;  // level i >= 1: [ns_i][2 ninter], rotated contiguous mod ns_{i-1}
  std::vector<std::vector<int>> antind;     // level i >= 1: [ns_i][2 ninter]
  std::vector<int> antcount;                // level i >= 1: longest anterpolation row
  std::vector<std::vector<cd>> shiftmul;    // level i < L-1: [4 children][ns_i]
  std::vector<std::vector<cd>> shiftloc;
  std::vector<std::vector<cd>> trans;       // level i >= 2: [49 offsets][ns_i]; offset (dy+3)*7 + dx+3

  // receiver ring (setup_mlfma.cpp:642-695)
  std::vector<double> interph;  // [numrx][ninter]
  std::vector<int> intindh;
  std::vector<double> anterph;  // [ns_0][2 ninter]
  std::vector<int> antindh;

  // orderings
  std::vector<cd> pos_tree;     // pixel centres in tree order (setup_mlfma.cpp:156-175)
  std::vector<int> unkmap;      // raster index -> tree index (setup_mlfma.cpp:177-185)
  std::vector<int> tree_of_blocked;    // blocked index -> tree index
  std::vector<int> raster_of_blocked;  // blocked index -> raster index
  std::vector<cd> pos_raster;   // pixel centres in raster order

  // near and trans (the Green's-function tables) are filled: by the host
  // (build_green_tables) or by the device at set-up (isg_tables_gpu.cu)
  bool green_ready = false;
};

// Builds every table; returns an empty string or an error message.  With
// with_green false the near-field blocks and translation operators (the
// tables that evaluate Bessel functions) are left for build_green_tables or
// the device.
std::string build_tables(int level, int box, double res, double k0, int beta, int ninter, int numrx, HostTables &t,
                         bool with_green = true);
// The near-field blocks and translation operators on the host (glibc jn, yn,
// j0, y0), as the reference computes them.
void build_green_tables(HostTables &t);

// integrate.cpp:15-41 for the displacement (posb - post) = (dx, dy).
cd green_entry(double k0, double res, double dx, double dy);

// Morton (tree) cluster index of raster cluster (row, col) at a level.
inline int tree_index(int row, int col, int lvl) {
  int idx = 0;
  for (int b = lvl - 1; b >= 0; b--) idx = idx * 4 + ((row >> b) & 1) * 2 + ((col >> b) & 1);
  return idx;
}

}  // namespace isg
