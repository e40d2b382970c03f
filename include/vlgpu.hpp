/*
 * vlgpu.hpp -- C++ drop-in layer over libvlgpu.so (vlgpu.h) with the
 * reference's own signatures for the acceleration path.  A Vlasiator build
 * that selects this library keeps its SpatialCell, VelocityMesh and
 * VelocityBlockContainer; the functions below read a cell's blocks, run the
 * hot path on the GPU and write the result back into the same containers, so
 * the rest of the code sees exactly what the reference's CPU functions leave:
 *
 *   vlgpu_dropin::map_1d               for  map_1d              (vlasovsolver/cpu_acc_map.hpp:30-32)
 *   vlgpu_dropin::gpu_accelerate_cells for  gpu_accelerate_cells (vlasovsolver/gpu_acc_semilag.hpp:31-35)
 *
 * Include it after the reference's common.h, object_wrapper.h and
 * spatial_cells/spatial_cell_wrapper.hpp: it names SpatialCell's members
 * (get_velocity_mesh, get_velocity_blocks, get_population, parameters,
 * derivativesBVOL), getObjectWrapper(), Parameters, bailout() and the
 * CellParams / bvolderivatives indices.  The functions are templates on the
 * cell type, so they compile against the reference's cell as they are.
 *
 * Results: the cell's blocks come back in ascending global-ID order (the
 * reference leaves them in its own local-ID order; the block set and the
 * values are what matter to every later step).  A column whose target blocks
 * come within the wall margin calls bailout() as map_1d does
 * (cpu_acc_map.cpp:325-338); any other library error also goes to bailout().
 * Device batches are kept per host thread and reused across calls.
 */
#ifndef VLGPU_HPP
#define VLGPU_HPP

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "vlgpu.h"

namespace vlgpu_dropin {

// Settings of the batches this layer creates: the remap arithmetic
// (vlgpu_batch_set_exact: 1 = the reference's operation order, bit-identical
// to map_1d; 0 = the fused default) and the CUDA device.
struct Settings {
   int exact = 0;
   int device = 0;
};
inline Settings& settings() {
   static Settings s;
   return s;
}

// A device batch reused by one host thread: recreated only when a call needs
// more cells or blocks than it holds, another mesh, other species settings
// or another arithmetic.  Unused cells of a call are left empty.
class BatchCache {
 public:
   ~BatchCache() {
      if (b_) vlgpu_batch_destroy(b_);
   }
   vlgpu_batch* get(const vlgpu_mesh& m, const vlgpu_params& p, uint32_t n_cells, uint64_t blocks) {
      const uint64_t need = 4 * blocks + 4096;  // room for the sweeps to add blocks
      const Settings& s = settings();
      if (b_ && (n_cells > cells_ || need > cap_ || !same(m, p) || exact_ != s.exact || device_ != s.device)) {
         vlgpu_batch_destroy(b_);
         b_ = nullptr;
      }
      if (!b_) {
         cells_ = std::max(n_cells, cells_);
         cap_ = std::max(need, cap_);
         if (vlgpu_batch_create(&m, &p, cells_, cap_, s.device, &b_) != VLGPU_OK) {
            b_ = nullptr;
            return nullptr;
         }
         vlgpu_batch_set_exact(b_, s.exact);
         mesh_ = m;
         params_ = p;
         exact_ = s.exact;
         device_ = s.device;
      }
      return b_;
   }
   uint32_t cells() const { return cells_; }

 private:
   bool same(const vlgpu_mesh& m, const vlgpu_params& p) const {
      for (int d = 0; d < 3; ++d)
         if (m.vmin[d] != mesh_.vmin[d] || m.vmax[d] != mesh_.vmax[d] || m.len[d] != mesh_.len[d]) return false;
      return p.charge == params_.charge && p.mass == params_.mass && p.min_value == params_.min_value &&
             p.add_width_v == params_.add_width_v && p.wall_margin == params_.wall_margin &&
             p.hall_minimum_rhoq == params_.hall_minimum_rhoq && p.ohm_gradpe == params_.ohm_gradpe;
   }
   vlgpu_batch* b_ = nullptr;
   uint32_t cells_ = 0;
   uint64_t cap_ = 0;
   vlgpu_mesh mesh_{};
   vlgpu_params params_{};
   int exact_ = -1;
   int device_ = -1;
};

inline BatchCache& thread_batch() {
   thread_local BatchCache cache;
   return cache;
}

// The velocity mesh of a population (vmesh::MeshParameters) as the library's.
template <class Cell>
vlgpu_mesh mesh_of(Cell* cell, uint32_t popID) {
   const auto* vm = cell->get_velocity_mesh(popID);
   vlgpu_mesh m{};
   for (int d = 0; d < 3; ++d) {
      m.vmin[d] = vm->getMeshMinLimits()[d];
      m.vmax[d] = vm->getMeshMaxLimits()[d];
      m.len[d] = vm->getGridLength()[d];
   }
   return m;
}

// The species and solver settings the hot path reads (object_wrapper.cpp,
// parameters.cpp), with the cell's own minValue.
template <class Cell>
vlgpu_params params_of(Cell* cell, uint32_t popID) {
   const auto& sp = getObjectWrapper().particleSpecies[popID];
   vlgpu_params p{};
   p.charge = sp.charge;
   p.mass = sp.mass;
   p.min_value = cell->getVelocityBlockMinValue(popID);
   p.add_width_v = (uint32_t)sp.sparseBlockAddWidthV;
   p.wall_margin = (uint32_t)Parameters::bailout_velocity_space_wall_margin;
   p.hall_minimum_rhoq = Parameters::hallMinimumRhoq;
   p.ohm_gradpe = (uint32_t)Parameters::ohmGradPeTerm;
   return p;
}

// The blocks of the cells, packed by cell in each cell's local-ID order.
template <class Cell>
void gather(const std::vector<Cell*>& cells, uint32_t popID, uint32_t n_slots, std::vector<uint64_t>& offsets,
            std::vector<uint32_t>& gids, std::vector<float>& data) {
   offsets.assign(n_slots + 1, 0);
   for (size_t c = 0; c < cells.size(); ++c) offsets[c + 1] = offsets[c] + cells[c]->get_velocity_mesh(popID)->size();
   for (size_t c = cells.size(); c < n_slots; ++c) offsets[c + 1] = offsets[c];
   gids.resize(offsets[n_slots]);
   data.resize(offsets[n_slots] * 64);
   for (size_t c = 0; c < cells.size(); ++c) {
      const auto* vm = cells[c]->get_velocity_mesh(popID);
      const auto* blocks = cells[c]->get_velocity_blocks(popID);
      const uint64_t n = vm->size();
      for (uint64_t l = 0; l < n; ++l) {
         gids[offsets[c] + l] = (uint32_t)vm->getGlobalID((vmesh::LocalID)l);
         const auto* src = blocks->getData((vmesh::LocalID)l);
         float* dst = &data[(offsets[c] + l) * 64];
         for (int i = 0; i < 64; ++i) dst[i] = (float)src[i];
      }
   }
}

// Replaces the population's blocks of the cell with n blocks (global IDs
// and 64 values each), setting each block's parameters from the mesh as
// SpatialCell::add_velocity_block does (spatial_cell_cpu.hpp:757-768).
template <class Cell>
void write_back(Cell* cell, uint32_t popID, const uint32_t* gids, const float* data, uint64_t n) {
   auto* vm = cell->get_velocity_mesh(popID);
   auto* blocks = cell->get_velocity_blocks(popID);
   vm->clear();
   blocks->clear();
   if (n == 0) return;
   std::vector<vmesh::GlobalID> g(gids, gids + n);
   if (!vm->push_back(g)) bailout(true, "vlgpu_dropin: the velocity mesh refused the blocks", __FILE__, __LINE__);
   const vmesh::LocalID first = blocks->push_back((uint32_t)n);
   for (uint64_t b = 0; b < n; ++b) {
      vm->getBlockInfo(g[b], blocks->getParameters(first + (vmesh::LocalID)b));
      auto* dst = blocks->getData(first + (vmesh::LocalID)b);
      for (int i = 0; i < 64; ++i) dst[i] = data[b * 64 + i];
   }
}

// Downloads every cell of the batch and writes the first cells.size() back.
template <class Cell>
void write_back_all(vlgpu_batch* b, const std::vector<Cell*>& cells, uint32_t popID, uint32_t n_slots) {
   std::vector<uint32_t> counts(n_slots);
   if (vlgpu_batch_block_counts(b, counts.data()) != VLGPU_OK)
      bailout(true, "vlgpu_dropin: vlgpu_batch_block_counts failed", __FILE__, __LINE__);
   uint64_t total = 0;
   for (uint32_t c : counts) total += c;
   std::vector<uint64_t> offsets(n_slots + 1);
   std::vector<uint32_t> gids(std::max<uint64_t>(total, 1));
   std::vector<float> data(std::max<uint64_t>(total, 1) * 64);
   if (vlgpu_batch_download(b, offsets.data(), gids.data(), data.data(), total) != VLGPU_OK)
      bailout(true, "vlgpu_dropin: vlgpu_batch_download failed", __FILE__, __LINE__);
   for (size_t c = 0; c < cells.size(); ++c)
      write_back(cells[c], popID, &gids[offsets[c]], &data[offsets[c] * 64], offsets[c + 1] - offsets[c]);
}

// The reference's bail-out for a column at the velocity-space wall, and for
// any other failed call.
inline void check(vlgpu_batch* b, int code, uint32_t n_cells, const char* what) {
   std::vector<uint32_t> status(n_cells);
   vlgpu_batch_status(b, status.data());
   for (uint32_t c = 0; c < n_cells; ++c) {
      if (status[c] & VLGPU_CELL_WALL)
         bailout(true, "vlgpu_dropin: target blocks within the velocity-space wall margin", __FILE__, __LINE__);
      else if (status[c])
         bailout(true, std::string("vlgpu_dropin: ") + what + ": cell status " + std::to_string(status[c]), __FILE__,
                 __LINE__);
   }
   if (code != VLGPU_OK) bailout(true, std::string("vlgpu_dropin: ") + what + " failed", __FILE__, __LINE__);
}

// map_1d (vlasovsolver/cpu_acc_map.hpp:30-32): one SLICE-3D 1D remap of the
// cell's population along `dimension` with the given intersections, blocks
// added and removed as the reference does; the cell's mesh and container
// hold the result on return.
template <class Cell>
bool map_1d(Cell* cell, const uint32_t popID, double intersection, double intersection_di, double intersection_dj,
            double intersection_dk, const uint32_t dimension) {
   const std::vector<Cell*> cells{cell};
   const vlgpu_mesh m = mesh_of(cell, popID);
   const vlgpu_params p = params_of(cell, popID);
   vlgpu_batch* b = thread_batch().get(m, p, 1, cell->get_velocity_mesh(popID)->size());
   if (!b) bailout(true, "vlgpu_dropin: vlgpu_batch_create failed", __FILE__, __LINE__);
   const uint32_t slots = thread_batch().cells();
   std::vector<uint64_t> offsets;
   std::vector<uint32_t> gids;
   std::vector<float> data;
   gather(cells, popID, slots, offsets, gids, data);
   int code = vlgpu_batch_upload(b, offsets.data(), gids.data(), data.data());
   if (code != VLGPU_OK) bailout(true, "vlgpu_dropin: vlgpu_batch_upload failed", __FILE__, __LINE__);
   std::vector<double> I(4 * (size_t)slots, 0.0);
   I[0] = intersection;
   I[1] = intersection_di;
   I[2] = intersection_dj;
   I[3] = intersection_dk;
   for (uint32_t c = 1; c < slots; ++c) I[4 * c + 3] = 1.0;  // empty cells
   code = vlgpu_map_1d(b, I.data(), dimension);
   check(b, code, 1, "vlgpu_map_1d");
   write_back_all(b, cells, popID, slots);
   return true;
}

// gpu_accelerate_cells (vlasovsolver/gpu_acc_semilag.hpp:31-35): the
// acceleration of the listed cells for one substep each (Population::
// subcycleDt) in map_order, as cpu_accelerate_cells does it
// (cpu_acc_semilag.cpp:45-130): the FP64 transform and intersections of every
// cell from its fields and its own first moments (stored in the population's
// intersection_* members as compute_cell_intersections stores them), then the
// three sweeps.  Block adjustment and moments stay with the caller, as in the
// reference.
template <class Grid, class IdList>
void gpu_accelerate_cells(Grid& mpiGrid, const IdList& acceleratedCells, const uint32_t popID,
                          const uint32_t map_order) {
   using CellPtr = decltype(mpiGrid[acceleratedCells[0]]);
   if (acceleratedCells.empty()) return;
   std::vector<CellPtr> cells;
   uint64_t blocks = 0;
   for (const auto id : acceleratedCells) {
      cells.push_back(mpiGrid[id]);
      blocks += cells.back()->get_velocity_mesh(popID)->size();
   }
   const vlgpu_mesh m = mesh_of(cells[0], popID);
   const vlgpu_params p = params_of(cells[0], popID);
   const uint32_t n = (uint32_t)cells.size();
   vlgpu_batch* b = thread_batch().get(m, p, n, blocks);
   if (!b) bailout(true, "vlgpu_dropin: vlgpu_batch_create failed", __FILE__, __LINE__);
   const uint32_t slots = thread_batch().cells();
   std::vector<uint64_t> offsets;
   std::vector<uint32_t> gids;
   std::vector<float> data;
   gather(cells, popID, slots, offsets, gids, data);
   int code = vlgpu_batch_upload(b, offsets.data(), gids.data(), data.data());
   if (code != VLGPU_OK) bailout(true, "vlgpu_dropin: vlgpu_batch_upload failed", __FILE__, __LINE__);
   // fields as compute_acceleration_transformation reads them (cpu_acc_transform.cpp:71-89)
   std::vector<vlgpu_cell_fields> fields(slots);
   std::vector<double> dt(slots, 0.0);
   for (uint32_t c = 0; c < slots; ++c) fields[c].B[2] = 1e-9;  // empty cells: any field
   for (uint32_t c = 0; c < n; ++c) {
      auto* sc = cells[c];
      fields[c].B[0] = sc->parameters[CellParams::BGBXVOL] + sc->parameters[CellParams::PERBXVOL];
      fields[c].B[1] = sc->parameters[CellParams::BGBYVOL] + sc->parameters[CellParams::PERBYVOL];
      fields[c].B[2] = sc->parameters[CellParams::BGBZVOL] + sc->parameters[CellParams::PERBZVOL];
      fields[c].curl[0] =
         sc->derivativesBVOL[bvolderivatives::dPERBZVOLdy] - sc->derivativesBVOL[bvolderivatives::dPERBYVOLdz];
      fields[c].curl[1] =
         sc->derivativesBVOL[bvolderivatives::dPERBXVOLdz] - sc->derivativesBVOL[bvolderivatives::dPERBZVOLdx];
      fields[c].curl[2] =
         sc->derivativesBVOL[bvolderivatives::dPERBYVOLdx] - sc->derivativesBVOL[bvolderivatives::dPERBXVOLdy];
      fields[c].egradpe[0] = sc->parameters[CellParams::EXGRADPE];
      fields[c].egradpe[1] = sc->parameters[CellParams::EYGRADPE];
      fields[c].egradpe[2] = sc->parameters[CellParams::EZGRADPE];
      dt[c] = sc->get_population(popID).subcycleDt;
   }
   code = vlgpu_compute_intersections(b, fields.data(), dt.data(), map_order);
   if (code != VLGPU_OK) bailout(true, "vlgpu_dropin: vlgpu_compute_intersections failed", __FILE__, __LINE__);
   std::vector<double> I(12 * (size_t)slots);
   vlgpu_batch_intersections(b, I.data());
   for (uint32_t c = 0; c < n; ++c) {
      auto& pop = cells[c]->get_population(popID);
      const double* x = &I[12 * (size_t)c];
      pop.intersection_x = x[0]; pop.intersection_x_di = x[1]; pop.intersection_x_dj = x[2]; pop.intersection_x_dk = x[3];
      pop.intersection_y = x[4]; pop.intersection_y_di = x[5]; pop.intersection_y_dj = x[6]; pop.intersection_y_dk = x[7];
      pop.intersection_z = x[8]; pop.intersection_z_di = x[9]; pop.intersection_z_dj = x[10]; pop.intersection_z_dk = x[11];
   }
   code = vlgpu_accelerate_with_intersections(b, I.data(), map_order);
   check(b, code, n, "vlgpu_accelerate_with_intersections");
   write_back_all(b, cells, popID, slots);
}

}  // namespace vlgpu_dropin

#endif  // VLGPU_HPP
