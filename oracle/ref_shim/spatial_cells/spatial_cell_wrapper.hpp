// Minimal stand-in for the reference's SpatialCell, used only when the
// reference's own hot-path sources are compiled as the parity oracle
// (oracle/build_ref.sh).  It owns one velocity mesh and one block container
// per population, built from the reference's own VelocityMesh and
// VelocityBlockContainer headers, and offers the member functions that
// cpu_acc_map.cpp, cpu_acc_sort_blocks.cpp, cpu_acc_load_blocks.cpp and the
// block-adjustment functions of spatial_cell_cpu.cpp call.  The inline
// helpers below follow their counterparts in spatial_cells/spatial_cell_cpu.hpp:
// add_velocity_block (:757-768) and remove_velocity_block (:826-850, "move the
// last block into the hole"), get_velocity_block_indices / get_velocity_block
// (:535-550), get_block_parameters (:445-462), get/set_max_r_dt
// (spatial_cell_cpu.cpp:322-352).  The block-adjustment member
// functions themselves (adjust_velocity_blocks, compute_block_has_content,
// update_velocity_block_content_lists, updateSparseMinValue) are the
// reference's own definitions, compiled from spatial_cell_cpu.cpp.
#pragma once
#include <array>
#include <deque>
#include <vector>
#include <dccrg.hpp>
#include <dccrg_cartesian_geometry.hpp>
#include <phiprof.hpp>
#include "../common.h"
#include "../memoryallocation.h"
#include "velocity_mesh_cpu.h"
#include "velocity_block_container.h"

namespace spatial_cell {

typedef std::array<vmesh::LocalID, 3> velocity_block_indices_t;

struct Population {
   vmesh::VelocityMesh* vmesh{nullptr};
   vmesh::VelocityBlockContainer* blockContainer{nullptr};
   Real velocityBlockMinValue{0};
   Real RHOLOSSADJUST{0};
   Real RHO{0};
   Real max_dt[2]{0, 0};  // species::MAXRDT, species::MAXVDT
   Real intersection_x{0}, intersection_x_di{0}, intersection_x_dj{0}, intersection_x_dk{0};
   Real intersection_y{0}, intersection_y_di{0}, intersection_y_dj{0}, intersection_y_dk{0};
   Real intersection_z{0}, intersection_z_di{0}, intersection_z_dj{0}, intersection_z_dk{0};
   Real subcycleDt{0};
   Population() {
      vmesh = new vmesh::VelocityMesh();
      blockContainer = new vmesh::VelocityBlockContainer();
   }
   ~Population() {
      delete vmesh;
      delete blockContainer;
   }
   Population(const Population&) = delete;
   Population& operator=(const Population&) = delete;
};

class SpatialCell {
 public:
   Real parameters[CellParams::N_SPATIAL_CELL_PARAMS];
   std::array<Real, bvolderivatives::N_BVOL_DERIVATIVES> derivativesBVOL{};
   std::deque<Population> populations;
   std::vector<vmesh::GlobalID>* velocity_block_with_content_list;
   std::vector<vmesh::GlobalID>* velocity_block_with_no_content_list;
   uint sysBoundaryFlag{sysboundarytype::NOT_SYSBOUNDARY};
   uint sysBoundaryLayer{0};

   explicit SpatialCell(size_t nPops = 1) {
      for (auto& p : parameters) p = 0;
      for (size_t i = 0; i < nPops; ++i) populations.emplace_back();
      velocity_block_with_content_list = new std::vector<vmesh::GlobalID>();
      velocity_block_with_no_content_list = new std::vector<vmesh::GlobalID>();
   }
   ~SpatialCell() {
      delete velocity_block_with_content_list;
      delete velocity_block_with_no_content_list;
   }
   SpatialCell(const SpatialCell&) = delete;
   SpatialCell& operator=(const SpatialCell&) = delete;

   vmesh::VelocityMesh* get_velocity_mesh(const size_t& popID) { return populations[popID].vmesh; }
   vmesh::VelocityBlockContainer* get_velocity_blocks(const size_t& popID) { return populations[popID].blockContainer; }
   Population& get_population(const uint popID) { return populations[popID]; }
   Real getVelocityBlockMinValue(const uint popID) const { return populations[popID].velocityBlockMinValue; }
   static vmesh::GlobalID invalid_global_id() { return vmesh::INVALID_GLOBALID; }
   static vmesh::LocalID invalid_local_id() { return vmesh::INVALID_LOCALID; }
   void debug_population_check(const uint) const {}
   void set_max_r_dt(const uint popID, const Real& value) { populations[popID].max_dt[0] = value; }
   const Real& get_max_r_dt(const uint popID) const { return populations[popID].max_dt[0]; }
   vmesh::LocalID get_number_of_velocity_blocks(const uint popID) const { return populations[popID].vmesh->size(); }
   vmesh::LocalID get_velocity_block_local_id(const vmesh::GlobalID& gid, const uint popID) const {
      return populations[popID].vmesh->getLocalID(gid);
   }
   velocity_block_indices_t get_velocity_block_indices(const uint popID, const vmesh::GlobalID block) {
      velocity_block_indices_t indices;
      populations[popID].vmesh->getIndices(block, indices[0], indices[1], indices[2]);
      return indices;
   }
   vmesh::GlobalID get_velocity_block(const uint popID, const velocity_block_indices_t indices) const {
      return populations[popID].vmesh->getGlobalID(indices[0], indices[1], indices[2]);
   }
   Real* get_block_parameters(const uint popID) { return populations[popID].blockContainer->getParameters(); }
   Real* get_block_parameters(const vmesh::LocalID& lid, const uint popID) {
      return populations[popID].blockContainer->getParameters(lid);
   }
   Realf* get_data(const uint popID) { return populations[popID].blockContainer->getData(); }
   Realf* get_data(const vmesh::LocalID lid, const uint popID) {
      return populations[popID].blockContainer->getData(lid);
   }
   bool add_velocity_block(const vmesh::GlobalID& gid, const uint popID) {
      Population& p = populations[popID];
      if (!p.vmesh->push_back(gid)) return false;
      const vmesh::LocalID lid = p.blockContainer->push_back_and_zero();
      p.vmesh->getBlockInfo(gid, p.blockContainer->getParameters(lid));
      return true;
   }
   void remove_velocity_block(const vmesh::GlobalID& gid, const uint popID) {
      if (gid == invalid_global_id()) return;
      Population& p = populations[popID];
      const vmesh::LocalID lid = p.vmesh->getLocalID(gid);
      if (lid == invalid_local_id()) return;
      const vmesh::LocalID last = p.vmesh->size() - 1;
      if (last == lid) {
         p.vmesh->pop();
         p.blockContainer->pop();
      } else {
         p.vmesh->move(last, lid);
         p.blockContainer->move(last, lid);
      }
   }

   // the reference's own definitions (spatial_cell_cpu.cpp), compiled by
   // oracle/build_ref.sh
   void adjust_velocity_blocks(const std::vector<SpatialCell*>& spatial_neighbors, const uint popID,
                               bool doDeleteEmptyBlocks = true);
   bool compute_block_has_content(const vmesh::LocalID& blockLID, const uint popID) const;
   void update_velocity_block_content_lists(const uint popID);
   void updateSparseMinValue(const uint popID);
};

}  // namespace spatial_cell

// the reference's own headers name the cell type unqualified
using spatial_cell::SpatialCell;
