// Declaration-only stand-in for the absent dccrg grid library (oracle builds
// only): the reference headers on the hot path name these types in
// declarations but the oracle never instantiates a grid.
#pragma once
namespace dccrg {
template <class Cell, class Geometry> class Dccrg;
class Cartesian_Geometry;
}  // namespace dccrg
