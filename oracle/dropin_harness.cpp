// Test harness for the C++ drop-in layer (include/vlgpu.hpp): instantiates
// vlgpu_dropin::map_1d and vlgpu_dropin::gpu_accelerate_cells with the
// stand-in SpatialCell and dccrg grid of the oracle build, so that the tests
// can run them beside the reference's own map_1d on copies of the same cells.
// Compiled by oracle/build_ref.sh together with ref_harness.cpp and the
// reference sources into oracle/_ref/libvlasov_ref_sp_dropin.so, which links
// libvlgpu.so (test infrastructure only).
#include <cstdint>
#include <vector>

#include "memoryallocation.h"
#include "object_wrapper.h"
#include "spatial_cells/spatial_cell_wrapper.hpp"
#include "vlgpu.hpp"

// the cell set of ref_harness.cpp
struct RefCells {
   std::vector<SpatialCell*> cells;
};

extern "C" {

void dropin_set_exact(int exact) { vlgpu_dropin::settings().exact = exact; }

// The species the drop-in layer reads from the object wrapper.
void dropin_set_species(double charge, double mass) {
   getObjectWrapper().particleSpecies[0].charge = charge;
   getObjectWrapper().particleSpecies[0].mass = mass;
}

// vlgpu_dropin::map_1d on every cell: intersections holds 4 doubles per cell.
void dropin_cells_map_1d(void* h, const double* intersections, uint32_t dimension) {
   RefCells* rc = (RefCells*)h;
   for (size_t c = 0; c < rc->cells.size(); ++c) {
      const double* I = intersections + 4 * c;
      vlgpu_dropin::map_1d(rc->cells[c], 0, I[0], I[1], I[2], I[3], dimension);
   }
}

// vlgpu_dropin::gpu_accelerate_cells on all cells of the set (dccrg ids
// c + 1), with the cells' background fields B (3 per cell; no perturbed field
// or derivatives) and substep lengths dt; the intersections it stored in the
// populations are returned in out12 (x, y, z; 4 each).
void dropin_cells_accelerate(void* h, const double* B, const double* dt, uint32_t map_order, double* out12) {
   RefCells* rc = (RefCells*)h;
   dccrg::Dccrg<SpatialCell, dccrg::Cartesian_Geometry> g;
   std::vector<CellID> ids;
   for (size_t c = 0; c < rc->cells.size(); ++c) {
      SpatialCell* sc = rc->cells[c];
      sc->parameters[CellParams::BGBXVOL] = B[3 * c + 0];
      sc->parameters[CellParams::BGBYVOL] = B[3 * c + 1];
      sc->parameters[CellParams::BGBZVOL] = B[3 * c + 2];
      sc->parameters[CellParams::PERBXVOL] = 0;
      sc->parameters[CellParams::PERBYVOL] = 0;
      sc->parameters[CellParams::PERBZVOL] = 0;
      sc->get_population(0).subcycleDt = dt[c];
      g.cells[c + 1] = sc;
      ids.push_back(c + 1);
   }
   vlgpu_dropin::gpu_accelerate_cells(g, ids, 0, map_order);
   for (size_t c = 0; c < rc->cells.size(); ++c) {
      const spatial_cell::Population& p = rc->cells[c]->get_population(0);
      const double v[12] = {p.intersection_x, p.intersection_x_di, p.intersection_x_dj, p.intersection_x_dk,
                            p.intersection_y, p.intersection_y_di, p.intersection_y_dj, p.intersection_y_dk,
                            p.intersection_z, p.intersection_z_di, p.intersection_z_dj, p.intersection_z_dk};
      for (int i = 0; i < 12; ++i) out12[12 * c + i] = v[i];
   }
}

}  // extern "C"
