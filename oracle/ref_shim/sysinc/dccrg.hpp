// Minimal stand-in for the absent dccrg grid library (oracle builds only):
// the reference's translation driver only looks cells up by id through
// operator[]; the oracle harness fills the map itself.
#pragma once
#include <algorithm>
#include <array>
#include <cstdint>
#include <map>
#include <set>
#include <unordered_set>
#include <unordered_map>
namespace dccrg {
class Cartesian_Geometry;
template <class Cell, class Geometry> class Dccrg {
 public:
   std::unordered_map<uint64_t, Cell*> cells;
   Cell* operator[](const uint64_t id) const {
      auto it = cells.find(id);
      return it == cells.end() ? nullptr : it->second;
   }
};
}  // namespace dccrg
