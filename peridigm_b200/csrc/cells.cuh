// Uniform cell grid shared by the bond-family search and the contact search.
// The grid only generates candidate pairs; each search's predicate decides.
#pragma once

#include "pd_internal.cuh"

namespace pdb {

struct Grid {
  double lo[3];
  double cell;
  int dims[3];
};

__device__ __forceinline__ int cell_coord(const Grid& g, double v, int k) {
  double q = floor((v - g.lo[k]) / g.cell);
  int c = (int)q;
  if (q < 0) c = 0;
  if (q >= g.dims[k]) c = g.dims[k] - 1;
  return c;
}

// Grid of cells of side >= reach over [lo, hi] (at most 4n+64 cells).
Grid make_grid(int64_t n, const double lo[3], const double hi[3], double reach);

// Bins n positions (xyz of double4) into grid g: sorted_idx lists the points
// cell by cell (ascending id within a cell), cell_start[q] the first entry of
// cell q (cell_start[ncell] = n).
// scratch (optional): the binning's temporaries kept between calls, so that
// a repeated search (contact, every search_frequency steps) allocates and
// frees no device memory once its buffers are large enough; sorted_idx and
// cell_start are then also only grown.
struct BinScratch {
  DBuf<int32_t> cid, idx, cid_s;
  DBuf<unsigned char> tmp;
};
int bin_points(pd_ctx* c, const double4* pos, int64_t n, const Grid& g, DBuf<int32_t>& sorted_idx,
               DBuf<int64_t>& cell_start, BinScratch* scratch = nullptr);

}  // namespace pdb
