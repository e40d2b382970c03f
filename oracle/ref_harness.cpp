// C entry points over the reference's own CPU hot-path code, used as the
// parity oracle and CPU baseline (test infrastructure only; built by
// oracle/build_ref.sh into oracle/_ref/, never linked into the product).
//
// The functions below build shim SpatialCells from flat (GID, data) arrays,
// call the reference's map_1d (vlasovsolver/cpu_acc_map.cpp:121-636) exactly
// as cpu_accelerate_cell does (vlasovsolver/cpu_acc_semilag.cpp:92-130), and
// read the resulting blocks back out.  The moment sums call the reference's
// blockVelocityFirstMoments / blockVelocitySecondMoments templates
// (vlasovsolver/arch_moments.h:83-155).
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include <omp.h>
#include <random>

#include "memoryallocation.h"
#include "object_wrapper.h"
#include "vlasovsolver/cpu_acc_map.hpp"
#include "vlasovsolver/arch_moments.h"
#include "vlasovsolver/cpu_trans_map_amr.hpp"
#include "vlasovsolver/cpu_trans_pencils.hpp"
#include "projects/project_density_part.h"

namespace spatial_cell {
// the reference's grid-level block adjustment (spatial_cells/block_adjust_cpu.cpp:33-117)
void update_velocity_block_content_lists(dccrg::Dccrg<SpatialCell, dccrg::Cartesian_Geometry>& mpiGrid,
                                         const std::vector<CellID>& cells, const uint popID);
void adjust_velocity_blocks_in_cells(dccrg::Dccrg<SpatialCell, dccrg::Cartesian_Geometry>& mpiGrid,
                                     const std::vector<CellID>& cellsToAdjust, const uint popID);
}  // namespace spatial_cell
// the reference's r-space time-step reduction (vlasovsolver/arch_dt.cpp:33-97)
void reduce_vlasov_dt(dccrg::Dccrg<SpatialCell, dccrg::Cartesian_Geometry>& mpiGrid, const std::vector<CellID>& cells,
                      Real (&dtMaxLocal)[3]);

using spatial_cell::SpatialCell;

uint Parameters::bailout_velocity_space_wall_margin = 1;
Real Parameters::maxSlAccelerationRotation = 25.0;
Real Parameters::hallMinimumRhoq = 1.60217653e-19;
uint Parameters::ohmGradPeTerm = 0;
bool Parameters::prepareForRebalance = false;
uint Parameters::tstep = 0;
bool Parameters::vlasovAccelerateMaxwellianBoundaries = false;

static ObjectWrapper g_objects;
ObjectWrapper& getObjectWrapper() { return g_objects; }

// The reference raises a global bail-out flag on fatal conditions
// (common.cpp:36-95); here every bail-out is counted so the caller can see it.
static int g_bailouts = 0;
void bailout(const bool condition, const std::string&, const char* const, const int) {
   if (condition) {
#pragma omp atomic
      g_bailouts++;
   }
}
void bailout(const bool condition, const std::string& m) { bailout(condition, m, "", 0); }
void bailout(const bool condition, const char* const f, const int l) { bailout(condition, "", f, l); }
void memory_purge() {}

static bool g_mesh_ready = false;
std::array<setOfPencils, 3> DimensionPencils;

extern "C" {

int ref_realf_size() { return (int)sizeof(Realf); }

// One velocity mesh: limits in m/s, grid length in blocks, WID cells per block.
int ref_init(const double vmin[3], const double vmax[3], const uint32_t grid_length[3], uint32_t wall_margin) {
   if (!g_mesh_ready) {
      vmesh::allocateMeshWrapper();
      vmesh::MeshParameters mp;
      mp.name = "mesh0";
      for (int d = 0; d < 3; ++d) {
         mp.meshLimits[2 * d] = vmin[d];
         mp.meshLimits[2 * d + 1] = vmax[d];
         mp.gridLength[d] = grid_length[d];
         mp.blockLength[d] = WID;
      }
      vmesh::host_getMeshWrapper()->velocityMeshesCreation->push_back(mp);
      vmesh::host_getMeshWrapper()->initVelocityMeshes(1);
      g_objects.particleSpecies.resize(1);
      g_mesh_ready = true;
   }
   Parameters::bailout_velocity_space_wall_margin = wall_margin;
   return 0;
}

// The initial condition of a list of blocks as the projects' fillPhaseSpace
// evaluates it (e.g. projects/Distributions/Distributions.cpp:161-178): the
// block's corner and cell size from VelocityMesh::getBlockInfo, and at each
// cell centre relative to the bulk velocity V the Maxwellian of temperature T
// or, with T_aniso (Tx, Ty, Tz) given, the tri-Maxwellian
// (projects/project.h:45-73).  Values in the cell order k*WID2 + j*WID + i.
void ref_fill_blocks(uint64_t n_blocks, const uint32_t* gids, const double V[3], double T, const double* T_aniso,
                     double rho, double mass, Realf* out) {
   SpatialCell cell(1);
   cell.get_velocity_mesh(0)->initialize(0);
   const vmesh::VelocityMesh* vm = cell.get_velocity_mesh(0);
#pragma omp parallel for schedule(static)
   for (uint64_t b = 0; b < n_blocks; ++b) {
      Real c[6];
      vm->getBlockInfo(gids[b], c);
      for (uint k = 0; k < WID; ++k)
         for (uint j = 0; j < WID; ++j)
            for (uint i = 0; i < WID; ++i) {
               const Real vx = c[0] + (i + 0.5) * c[3] - V[0];
               const Real vy = c[1] + (j + 0.5) * c[4] - V[1];
               const Real vz = c[2] + (k + 0.5) * c[5] - V[2];
               out[b * WID3 + k * WID2 + j * WID + i] =
                   T_aniso ? projects::TriMaxwellianPhaseSpaceDensity(vx, vy, vz, T_aniso[0], T_aniso[1], T_aniso[2],
                                                                      rho, mass)
                           : projects::MaxwellianPhaseSpaceDensity(vx, vy, vz, T, rho, mass);
            }
   }
}

int ref_bailouts() { return g_bailouts; }
void ref_reset_bailouts() { g_bailouts = 0; }

// ---- a set of cells kept alive across calls (for timing without set-up) ----
struct RefCells {
   std::vector<SpatialCell*> cells;
};

void* ref_cells_create(uint32_t n_cells, const uint64_t* offsets, const uint32_t* gids, const Realf* data,
                       const double* min_values) {
   RefCells* rc = new RefCells();
   rc->cells.resize(n_cells);
#pragma omp parallel for schedule(dynamic, 16)
   for (uint32_t c = 0; c < n_cells; ++c) {
      SpatialCell* sc = new SpatialCell(1);
      sc->get_velocity_mesh(0)->initialize(0);
      sc->populations[0].velocityBlockMinValue = min_values[c];
      sc->parameters[CellParams::CELLID] = c + 1;
      const uint64_t b0 = offsets[c], b1 = offsets[c + 1];
      for (uint64_t b = b0; b < b1; ++b) {
         if (!sc->add_velocity_block(gids[b], 0)) continue;
         const vmesh::LocalID lid = sc->get_velocity_mesh(0)->getLocalID(gids[b]);
         std::memcpy(sc->get_velocity_blocks(0)->getData(lid), data + b * WID3, sizeof(Realf) * WID3);
      }
      rc->cells[c] = sc;
   }
   return rc;
}

void ref_cells_destroy(void* h) {
   RefCells* rc = (RefCells*)h;
   for (auto* c : rc->cells) delete c;
   delete rc;
}

uint32_t ref_cells_count(void* h) { return (uint32_t)((RefCells*)h)->cells.size(); }

uint64_t ref_cells_block_count(void* h, uint32_t c) { return ((RefCells*)h)->cells[c]->get_velocity_mesh(0)->size(); }

// Copies cell c's blocks out in the container's local-ID order.
uint64_t ref_cells_extract(void* h, uint32_t c, uint32_t* gids, Realf* data, uint64_t cap) {
   SpatialCell* sc = ((RefCells*)h)->cells[c];
   const uint64_t n = sc->get_velocity_mesh(0)->size();
   if (n > cap) return n;
   for (uint64_t lid = 0; lid < n; ++lid) {
      gids[lid] = sc->get_velocity_mesh(0)->getGlobalID(lid);
      std::memcpy(data + lid * WID3, sc->get_velocity_blocks(0)->getData(lid), sizeof(Realf) * WID3);
   }
   return n;
}

// One 1D sweep on every cell: intersections holds 4 doubles per cell
// (intersection, di, dj, dk) for this dimension.
void ref_cells_map_1d(void* h, const double* intersections, uint32_t dimension, int nthreads) {
   RefCells* rc = (RefCells*)h;
   if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
   for (size_t c = 0; c < rc->cells.size(); ++c) {
      const double* I = intersections + 4 * c;
      map_1d(rc->cells[c], 0, I[0], I[1], I[2], I[3], dimension);
   }
}

// Three sweeps per cell in map_order 0 (XYZ), 1 (YZX) or 2 (ZXY), as
// cpu_accelerate_cell does; intersections holds 12 doubles per cell ordered
// x(4), y(4), z(4).
void ref_cells_accelerate(void* h, const double* intersections, uint32_t map_order, int nthreads) {
   RefCells* rc = (RefCells*)h;
   static const uint32_t orders[3][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}};
   if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
   for (size_t c = 0; c < rc->cells.size(); ++c) {
      const double* I = intersections + 12 * c;
      for (int s = 0; s < 3; ++s) {
         const uint32_t d = orders[map_order % 3][s];
         map_1d(rc->cells[c], 0, I[4 * d + 0], I[4 * d + 1], I[4 * d + 2], I[4 * d + 3], d);
      }
   }
}

// First moments (n, nVx, nVy, nVz) and, about the given bulk velocity, the
// six second moments of cell c, with the reference's own reduction templates.
void ref_cells_moments(void* h, uint32_t c, const double* bulk_v, double* first4, double* second6) {
   SpatialCell* sc = ((RefCells*)h)->cells[c];
   const uint n = sc->get_velocity_mesh(0)->size();
   Real a1[4] = {0, 0, 0, 0};
   Real a2[6] = {0, 0, 0, 0, 0, 0};
   if (n > 0) {
      blockVelocityFirstMoments(sc->get_velocity_blocks(0), a1, n);
      blockVelocitySecondMoments(sc->get_velocity_blocks(0), (Real)bulk_v[0], (Real)bulk_v[1], (Real)bulk_v[2], a2, n);
   }
   for (int i = 0; i < 4; ++i) first4[i] = a1[i];
   for (int i = 0; i < 6; ++i) second6[i] = a2[i];
}

// One acceleration step per cell, the body of calculateAcceleration for one
// substep (vlasovsolver/vlasovmover.cpp:410-475) without the block
// adjustment: first moments with the reference's reduction template give the
// pivot velocity (calculateMoments_V), the FP64 transform and intersections
// come from the oracle's restatement (the reference needs Eigen for them), and
// the reference's map_1d runs three times in map_order.  B: 3 doubles per cell;
// dt: one per cell.
void orc_acceleration_transform(const double B[3], const double curl_terms[3], double rhoq_v, const double V[3],
                                const double egradpe[3], double q, double m, double dt, double hall_min_rhoq,
                                int ohm_gradpe, double mu0, double out_L[9], double out_t[3]);
struct orc_mesh_c {
   double vmin[3];
   double vmax[3];
   uint32_t len[3];
};
void orc_cell_intersections(const double fwd_L[9], const double fwd_t[3], const orc_mesh_c* m, uint32_t map_order,
                            double out12[12]);

void ref_cells_accelerate_step(void* h, const double* B, const double* dt, uint32_t map_order, double charge,
                               double mass, int nthreads) {
   RefCells* rc = (RefCells*)h;
   static const uint32_t orders[3][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}};
   if (nthreads > 0) omp_set_num_threads(nthreads);
   const vmesh::MeshParameters& mp = (*vmesh::host_getMeshWrapper()->velocityMeshes)[0];
   orc_mesh_c om;
   for (int d = 0; d < 3; ++d) {
      om.vmin[d] = mp.meshMinLimits[d];
      om.vmax[d] = mp.meshMaxLimits[d];
      om.len[d] = mp.gridLength[d];
   }
#pragma omp parallel for schedule(dynamic, 1)
   for (size_t c = 0; c < rc->cells.size(); ++c) {
      SpatialCell* sc = rc->cells[c];
      const uint n = sc->get_velocity_mesh(0)->size();
      Real a[4] = {0, 0, 0, 0};
      if (n > 0) blockVelocityFirstMoments(sc->get_velocity_blocks(0), a, n);
      const double rhom = a[0] * mass;
      const double V[3] = {rhom != 0 ? (a[1] * mass) / rhom : 0.0, rhom != 0 ? (a[2] * mass) / rhom : 0.0,
                           rhom != 0 ? (a[3] * mass) / rhom : 0.0};
      const double zero[3] = {0, 0, 0};
      double L[9], t[3], I[12];
      orc_acceleration_transform(B + 3 * c, zero, a[0] * charge, V, zero, charge, mass, dt[c],
                                 Parameters::hallMinimumRhoq, 0, 1.25663706e-6, L, t);
      orc_cell_intersections(L, t, &om, map_order % 3, I);
      for (int s = 0; s < 3; ++s) {
         const uint32_t d = orders[map_order % 3][s];
         map_1d(sc, 0, I[4 * d + 0], I[4 * d + 1], I[4 * d + 2], I[4 * d + 3], d);
      }
   }
}

// Block adjustment of every cell of the set as adjustVelocityBlocks does it
// (grid.cpp:775-817): the reference's own update_velocity_block_content_lists
// (block_adjust_cpu.cpp:33-53, with updateSparseMinValue and
// compute_block_has_content, spatial_cell_cpu.cpp:290-316, 675-727) for all
// cells first, then adjust_velocity_blocks_in_cells (block_adjust_cpu.cpp:
// 55-117) calling SpatialCell::adjust_velocity_blocks (spatial_cell_cpu.cpp:
// 179-273).  Cell c has dccrg id c+1; neighbors holds n_per_cell cell indices
// per cell (-1: none) -- the cell's NEAREST neighbourhood -- or is null (no
// spatial neighbours).  The species' minValue and blockAddWidthV are set from
// min_value and add_width; rho_loss gets each cell's RHOLOSSADJUST added by
// this call.
static void adjust_cells(RefCells* rc, const int32_t* neighbors, uint32_t n_per_cell, double* rho_loss) {
   dccrg::Dccrg<SpatialCell, dccrg::Cartesian_Geometry> g;
   std::vector<CellID> cells;
   std::vector<double> before(rc->cells.size());
   for (size_t c = 0; c < rc->cells.size(); ++c) {
      g.cells[c + 1] = rc->cells[c];
      cells.push_back(c + 1);
      before[c] = rc->cells[c]->populations[0].RHOLOSSADJUST;
      if (neighbors) {
         auto& list = g.neighbor_lists[c + 1];
         for (uint32_t q = 0; q < n_per_cell; ++q) {
            const int32_t n = neighbors[(size_t)c * n_per_cell + q];
            if (n >= 0) list.push_back({(uint64_t)n + 1, std::array<int, 4>{0, 0, 0, 0}});
         }
      }
   }
   spatial_cell::update_velocity_block_content_lists(g, cells, 0);
   spatial_cell::adjust_velocity_blocks_in_cells(g, cells, 0);
   if (rho_loss)
      for (size_t c = 0; c < rc->cells.size(); ++c)
         rho_loss[c] = rc->cells[c]->populations[0].RHOLOSSADJUST - before[c];
}

void ref_cells_adjust(void* h, const int32_t* neighbors, uint32_t n_per_cell, double min_value, int add_width,
                      int conserve_mass, int nthreads, double* rho_loss) {
   RefCells* rc = (RefCells*)h;
   if (nthreads > 0) omp_set_num_threads(nthreads);
   species::Species& sp = getObjectWrapper().particleSpecies[0];
   sp.sparseMinValue = min_value;
   sp.sparseBlockAddWidthV = add_width;
   sp.sparse_conserve_mass = conserve_mass != 0;
   sp.sparseDynamicAlgorithm = 0;
   adjust_cells(rc, neighbors, n_per_cell, rho_loss);
}

// First moments and, about the bulk velocity, second moments of every cell
// with the reference's reduction templates (arch_moments.h:83-155), as
// calculateMoments_V(..., computeSecond=true) forms them; out: 10 per cell
// (n, n V (3), sum f (v - V)_a (v - V)_b (6)); may be null (timing only).
static void moments_cells(RefCells* rc, double* out) {
#pragma omp parallel for schedule(dynamic, 4)
   for (size_t c = 0; c < rc->cells.size(); ++c) {
      SpatialCell* sc = rc->cells[c];
      const uint n = sc->get_velocity_mesh(0)->size();
      Real a1[4] = {0, 0, 0, 0};
      Real a2[6] = {0, 0, 0, 0, 0, 0};
      if (n > 0) {
         blockVelocityFirstMoments(sc->get_velocity_blocks(0), a1, n);
         const Real V[3] = {a1[0] != 0 ? a1[1] / a1[0] : 0, a1[0] != 0 ? a1[2] / a1[0] : 0,
                            a1[0] != 0 ? a1[3] / a1[0] : 0};
         blockVelocitySecondMoments(sc->get_velocity_blocks(0), V[0], V[1], V[2], a2, n);
      }
      if (out) {
         for (int i = 0; i < 4; ++i) out[10 * c + i] = a1[i];
         for (int i = 0; i < 6; ++i) out[10 * c + 4 + i] = a2[i];
      }
   }
}

// The content flag of every block of cell c in local-ID order, as the
// reference's compute_block_has_content gives it (spatial_cell_cpu.cpp:290-316).
uint64_t ref_cells_content(void* h, uint32_t c, uint8_t* flags, uint64_t cap) {
   SpatialCell* sc = ((RefCells*)h)->cells[c];
   const uint64_t n = sc->get_velocity_mesh(0)->size();
   if (n > cap) return n;
   for (uint64_t lid = 0; lid < n; ++lid) flags[lid] = sc->compute_block_has_content((vmesh::LocalID)lid, 0) ? 1 : 0;
   return n;
}

// The r-space time-step limit of every cell of the set with the reference's
// own reduce_vlasov_dt (vlasovsolver/arch_dt.cpp:33-97): the minimum over the
// cell's blocks of dx/|v| at the centres of the block's first and last
// cells.  dx: the cell sizes (DX, DY, DZ); r_dt gets each cell's MAXRDT;
// returns the reduction over all cells (dtMaxLocal[0]).
double ref_cells_max_r_dt(void* h, const double dx[3], double* r_dt) {
   RefCells* rc = (RefCells*)h;
   dccrg::Dccrg<SpatialCell, dccrg::Cartesian_Geometry> g;
   std::vector<CellID> cells;
   for (size_t c = 0; c < rc->cells.size(); ++c) {
      SpatialCell* sc = rc->cells[c];
      sc->parameters[CellParams::DX] = dx[0];
      sc->parameters[CellParams::DY] = dx[1];
      sc->parameters[CellParams::DZ] = dx[2];
      sc->parameters[CellParams::MAXVDT] = 0;
      g.cells[c + 1] = sc;
      cells.push_back(c + 1);
   }
   Real dt_max[3] = {std::numeric_limits<Real>::max(), std::numeric_limits<Real>::max(),
                     std::numeric_limits<Real>::max()};
   reduce_vlasov_dt(g, cells, dt_max);
   for (size_t c = 0; c < rc->cells.size(); ++c) r_dt[c] = rc->cells[c]->parameters[CellParams::MAXRDT];
   return dt_max[0];
}

// The dimension order of time step `tstep`, drawn as calculateAcceleration
// draws it for every subcycle of that step (vlasovsolver/vlasovmover.cpp:
// 422-426): a default_random_engine seeded with the step number and one
// uniform_int_distribution<>(0, 2) draw, with this compiler's standard library.
uint32_t ref_map_order(uint32_t tstep) {
   std::default_random_engine rndState;
   rndState.seed(tstep);
   return (uint32_t)std::uniform_int_distribution<>(0, 2)(rndState);
}

// One full acceleration step of every cell of the set, the body of
// calculateAcceleration for one population and one subcycle
// (vlasovsolver/vlasovmover.cpp:410-475, 564-569): pivot moments, geometry and
// map_1d x3 (ref_cells_accelerate_step), then adjustVelocityBlocks
// (grid.cpp:775-817: content lists of all cells, then each cell with the
// NEAREST neighbours given in `neighbors`, n_per_cell per cell, or none), then
// calculateMoments_V with the second moments.  moments_out: 10 per cell or null.
void ref_cells_full_step(void* h, const double* B, const double* dt, uint32_t map_order, double charge, double mass,
                         const int32_t* neighbors, uint32_t n_per_cell, int nthreads, double* moments_out) {
   RefCells* rc = (RefCells*)h;
   ref_cells_accelerate_step(h, B, dt, map_order, charge, mass, nthreads);
   adjust_cells(rc, neighbors, n_per_cell, nullptr);
   moments_cells(rc, moments_out);
}

void ref_cells_translate(void* h, const uint32_t grid[3], uint32_t dimension, double dt, double dz, int nthreads);

// One full Vlasov step of a uniform periodic grid (cells x fastest) in the
// reference's main-loop order: calculateSpatialTranslation (trans_map_1d_amr
// along z, x, y, vlasovmover.cpp:65-381) and the "_R" moments, then the full
// acceleration step above with the spatial neighbours in the adjustment.
// moments_out (n_cells x 10, as ref_cells_full_step) and rho_loss (the
// RHOLOSSADJUST each cell gained in the step) may be null.
void ref_cells_vlasov_step(void* h, const uint32_t grid[3], const double dx[3], const double* B, double dt,
                           uint32_t map_order, double charge, double mass, const int32_t* neighbors,
                           uint32_t n_per_cell, int nthreads, double* moments_out, double* rho_loss) {
   RefCells* rc = (RefCells*)h;
   static const uint32_t dims[3] = {2, 0, 1};
   for (uint32_t q = 0; q < 3; ++q) ref_cells_translate(h, grid, dims[q], dt, dx[dims[q]], nthreads);
   moments_cells(rc, nullptr);
   std::vector<double> dts(rc->cells.size(), dt);
   ref_cells_accelerate_step(h, B, dts.data(), map_order, charge, mass, nthreads);
   adjust_cells(rc, neighbors, n_per_cell, rho_loss);
   moments_cells(rc, moments_out);
}

int ref_max_threads() { return omp_get_max_threads(); }

// Translation of a uniform periodic grid along one dimension with the
// reference's own trans_map_1d_amr (vlasovsolver/cpu_trans_map_amr.cpp:214-443).
// Cells are x fastest and hold the blocks of the cell set `h` (cell c has
// dccrg id c+1).  One pencil per grid line, padded with the periodic
// neighbours (two on each side, the outer ones pure sources), as the
// reference's pencil builder produces for a periodic dimension.
void ref_cells_translate(void* h, const uint32_t grid[3], uint32_t dimension, double dt, double dz, int nthreads) {
   RefCells* rc = (RefCells*)h;
   if (nthreads > 0) omp_set_num_threads(nthreads);
   dccrg::Dccrg<SpatialCell, dccrg::Cartesian_Geometry> g;
   std::vector<CellID> local;
   for (size_t c = 0; c < rc->cells.size(); ++c) {
      g.cells[c + 1] = rc->cells[c];
      local.push_back(c + 1);
   }
   const uint32_t nx = grid[0], ny = grid[1], nz = grid[2];
   const uint32_t N = grid[dimension];
   const uint64_t stride = dimension == 0 ? 1 : (dimension == 1 ? nx : (uint64_t)nx * ny);
   const uint32_t n_lines = (uint32_t)(rc->cells.size() / N);
   setOfPencils& P = DimensionPencils[dimension];
   P.removeAllPencils();
   for (uint32_t p = 0; p < n_lines; ++p) {
      uint64_t c0;
      if (dimension == 0) c0 = (uint64_t)p * nx;
      else if (dimension == 1) c0 = (uint64_t)(p % nx) + (uint64_t)nx * ny * (p / nx);
      else c0 = p;
      std::vector<CellID> ids;
      for (uint32_t x = 0; x < N; ++x) ids.push_back(c0 + x * stride + 1);
      P.addPencil(ids, 0.0, 0.0, false, std::vector<uint>());
      const uint start = P.idsStart.back(), L = P.lengthOfPencils.back();
      for (int s = 0; s < VLASOV_STENCIL_WIDTH; ++s) {
         P.ids[start + s] = c0 + ((N - VLASOV_STENCIL_WIDTH + s) % N) * stride + 1;
         P.ids[start + L - VLASOV_STENCIL_WIDTH + s] = c0 + ((uint64_t)s % N) * stride + 1;
      }
      for (uint q = 0; q < L; ++q) {
         P.sourceDZ[start + q] = (Realf)dz;
         P.targetRatios[start + q] = (q == 0 || q + 1 == L) ? 0.0 : 1.0;
      }
   }
   P.binPencils();
   std::vector<uint> nPencils(local.size() + 1, 0);
   trans_map_1d_amr(g, local, std::vector<CellID>(), nPencils, dimension, (Realf)dt, 0);
   (void)nz;
}

}  // extern "C"
