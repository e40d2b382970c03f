// Minimal stand-in for the reference's SpatialCell, used only when the
// reference's own acceleration sources are compiled as the parity oracle
// (oracle/build_ref.sh).  It owns one velocity mesh and one block container
// per population, built from the reference's own VelocityMesh and
// VelocityBlockContainer headers, and offers exactly the member functions
// that cpu_acc_map.cpp, cpu_acc_sort_blocks.cpp and cpu_acc_load_blocks.cpp
// call.  remove_velocity_block follows the reference's "move the last block
// into the hole" rule (spatial_cells/spatial_cell_cpu.hpp:826-850).
#pragma once
#include <array>
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
   std::vector<Population*> populations;

   explicit SpatialCell(size_t nPops = 1) {
      for (auto& p : parameters) p = 0;
      for (size_t i = 0; i < nPops; ++i) populations.push_back(new Population());
   }
   ~SpatialCell() {
      for (auto* p : populations) delete p;
   }
   SpatialCell(const SpatialCell&) = delete;
   SpatialCell& operator=(const SpatialCell&) = delete;

   vmesh::VelocityMesh* get_velocity_mesh(const size_t& popID) { return populations[popID]->vmesh; }
   vmesh::VelocityBlockContainer* get_velocity_blocks(const size_t& popID) { return populations[popID]->blockContainer; }
   Population& get_population(const uint popID) { return *populations[popID]; }
   Real getVelocityBlockMinValue(const uint popID) const { return populations[popID]->velocityBlockMinValue; }
   static vmesh::GlobalID invalid_global_id() { return vmesh::INVALID_GLOBALID; }
   static vmesh::LocalID invalid_local_id() { return vmesh::INVALID_LOCALID; }
   vmesh::LocalID get_velocity_block_local_id(const vmesh::GlobalID& gid, const uint popID) const {
      return populations[popID]->vmesh->getLocalID(gid);
   }
   Realf* get_data(const uint popID) { return populations[popID]->blockContainer->getData(); }
   Realf* get_data(const vmesh::LocalID lid, const uint popID) {
      return populations[popID]->blockContainer->getData(lid);
   }
   bool add_velocity_block(const vmesh::GlobalID& gid, const uint popID) {
      Population& p = *populations[popID];
      if (!p.vmesh->push_back(gid)) return false;
      const vmesh::LocalID lid = p.blockContainer->push_back_and_zero();
      p.vmesh->getBlockInfo(gid, p.blockContainer->getParameters(lid));
      return true;
   }
   void remove_velocity_block(const vmesh::GlobalID& gid, const uint popID) {
      if (gid == invalid_global_id()) return;
      Population& p = *populations[popID];
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
};

}  // namespace spatial_cell

// the reference's own headers name the cell type unqualified
using spatial_cell::SpatialCell;
