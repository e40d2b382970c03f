// Minimal stand-in for the absent dccrg grid library (oracle builds only):
// the reference's translation driver looks cells up by id through
// operator[], and its block-adjustment driver asks for a cell's neighbour
// list (get_neighbors_of, pairs of neighbour id and direction); the oracle
// harness fills both itself.
#pragma once
#include <algorithm>
#include <array>
#include <cstdint>
#include <map>
#include <set>
#include <unordered_set>
#include <unordered_map>
#include <utility>
#include <vector>
namespace dccrg {
class Cartesian_Geometry;
template <class Cell, class Geometry> class Dccrg {
 public:
   std::unordered_map<uint64_t, Cell*> cells;
   std::unordered_map<uint64_t, std::vector<std::pair<uint64_t, std::array<int, 4>>>> neighbor_lists;
   Cell* operator[](const uint64_t id) const {
      auto it = cells.find(id);
      return it == cells.end() ? nullptr : it->second;
   }
   const std::vector<std::pair<uint64_t, std::array<int, 4>>>* get_neighbors_of(const uint64_t id, int) const {
      static const std::vector<std::pair<uint64_t, std::array<int, 4>>> none;
      auto it = neighbor_lists.find(id);
      return it == neighbor_lists.end() ? &none : &it->second;
   }
};
}  // namespace dccrg
