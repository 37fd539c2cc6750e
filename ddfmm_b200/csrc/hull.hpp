// Extreme points of a 3-D point set (the vertices of its convex hull).
//
// The reference's precompute takes the vertices of MATLAB convhulln (Qhull)
// triangulations as the points that a skeleton must keep
// (matlab/aug3d_hghdata.m:112-113,129-130,166-167).  Qhull merges coplanar
// facets, so its vertices are the extreme points: corners, not points in the
// middle of a flat face or a straight edge.  hull_vertices returns the same
// set, computed as an incremental (beneath-beyond) hull with a relative
// tolerance, then keeping the hull vertices whose incident facet normals span
// all three dimensions.
#pragma once
#include <vector>

namespace ddfmm {

// pts: 3 x n, coordinate fastest (x[3k + d]).  Returns the indices of the
// extreme points in ascending order; throws if the points span no volume.
std::vector<int> hull_vertices(const std::vector<double>& pts);

}  // namespace ddfmm
