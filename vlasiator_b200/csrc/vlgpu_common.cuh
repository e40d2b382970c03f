// Shared device-side definitions for the vlgpu kernels (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/vlgpu.h"

namespace vlgpu {

constexpr int WID = 4;
constexpr int WID2 = 16;
constexpr int WID3 = 64;
constexpr int MAX_LEN = 96;         // blocks per mesh axis supported by the 3-word column masks
constexpr int MAX_PLANE = 96 * 96;  // transverse plane entries

// The moments split a cell's blocks into at most this many parts, each
// summed by one warp into MOM_SUMS_PER_PART doubles of a work array.
constexpr int MOM_PARTS_PER_CELL = 64;
constexpr int MOM_SUMS_PER_PART = 10;

// Per-cell state of one batch, indexed by cell.
struct CellSlot {
   uint32_t off;     // first block in the current pool
   uint32_t count;   // number of blocks
};

// One column set of one sweep: all blocks of a cell that share the two
// transverse block indices.  Built by the columnize kernel, consumed by the
// remap kernel.
struct ColumnSet {
   uint32_t cell;
   uint32_t si, sj;     // transverse block indices in the swapped frame
   uint32_t src_pos;    // first entry in the permutation array (absolute)
   uint32_t dst_pos;    // first output block (absolute, destination pool)
   uint32_t src_mask[3];
   uint32_t tgt_mask[3];
};

// Per-cell sweep parameters, already converted to Realf and swapped into the
// frame where the sweep dimension is k (cpu_acc_map.cpp:127-199).
struct SweepCell {
   float intersection, di, dj, dk;
   float threshold;
   uint32_t flags;  // SWEEP_PASS
};

// The cell is not accelerated in this step (its substep length is zero, as
// for a cell that has finished its subcycles, vlasovmover.cpp:527-556): the
// sweep passes its blocks through unchanged.
constexpr uint32_t SWEEP_PASS = 1u;

// Per-cell sweep parameters of one dimension from the four doubles
// (intersection, di, dj, dk) the reference stores per population, cast to
// Realf and swapped into the frame where the sweep dimension is k
// (cpu_acc_map.cpp:127-176).  Every entry point that sweeps uses this one
// conversion.
inline SweepCell make_sweep_cell(const double* I, uint32_t dim, double min_value) {
   SweepCell s{};
   float di = (float)I[1], dj = (float)I[2], dk = (float)I[3];
   if (dim == 0) { const float t = di; di = dk; dk = t; }
   if (dim == 1) { const float t = dj; dj = dk; dk = t; }
   s.intersection = (float)I[0];
   s.di = di;
   s.dj = dj;
   s.dk = dk;
   s.threshold = (float)min_value;
   return s;
}

// Mesh constants used on the device (cell size and origin already in Realf),
// with the reciprocals of block_xyz (zero: plain division).
struct MeshDev {
   uint32_t len[3];
   float dv[3];
   float vmin[3];
   uint32_t m0 = 0, m1 = 0;
};

// Reciprocals for the block-index decomposition of block_xyz: floor(n / d) =
// umulhi(n, floor(2^32 / d) + 1) holds exactly for n < 2^32 / d (division by
// invariant integers, Granlund and Montgomery 1994), so they are set only when
// every block ID n < L0 L1 L2 satisfies it for d = L0 and every n / L0 for
// d = L1.
inline void set_block_reciprocals(MeshDev& m) {
   const uint64_t L0 = m.len[0], L1 = m.len[1], L2 = m.len[2];
   const uint64_t two32 = 1ull << 32;
   m.m0 = m.m1 = 0;
   if (L0 < 2 || L1 < 2 || L0 * L1 * L2 * L0 >= two32 || L1 * L2 * L1 >= two32) return;
   m.m0 = (uint32_t)(two32 / L0 + 1);
   m.m1 = (uint32_t)(two32 / L1 + 1);
}

// x = g mod L0, y = (g / L0) mod L1, z = g / (L0 L1) of block ID g.
__device__ __forceinline__ void block_xyz(const MeshDev& m, uint32_t g, uint32_t& x, uint32_t& y, uint32_t& z) {
   if (m.m0) {
      const uint32_t q0 = __umulhi(g, m.m0);
      x = g - q0 * m.len[0];
      z = __umulhi(q0, m.m1);
      y = q0 - z * m.len[1];
   } else {
      const uint32_t q0 = g / m.len[0];
      x = g - q0 * m.len[0];
      z = q0 / m.len[1];
      y = q0 - z * m.len[1];
   }
}

// Content mask of one cell for the block adjustment on a grid: the (y, z)
// bounding box of its content blocks (y1 < 0: none) and the offset of its
// x-mask rows (3 words per row) in the mask pool, or 0xffffffff when the rows
// were not stored (the cell's block list is read instead).
// The velocity mesh in FP64 for the moment sums: minimum, block size and
// cell size per dimension, and the species' mass and charge.
struct MomentFrame {
   double vmin[3], bs[3], dv[3];
   double mass, charge;
};

struct MaskRec {
   int32_t y0, y1, z0, z1;
   uint32_t off;
   uint32_t pad[3];
};

// Counters of one sweep, zeroed before the columnize launch.
struct SweepCounters {
   uint32_t n_sets;
   uint32_t dst_top;
   uint32_t work;
   uint32_t overflow;
   uint32_t cell_next;  // warp-per-cell kernels (columnize, adjustment): next cell a warp takes
   uint32_t n_wide;     // cells those kernels left to their CTA-per-cell forms
};

// Running totals kept on the device across sweeps (never reset by a sweep).
struct BatchStats {
   unsigned long long src_blocks;  // source blocks entering sweeps
   unsigned long long dst_blocks;  // blocks written by sweeps
   unsigned long long sweeps;      // cell-sweeps performed
   unsigned long long sets;        // column sets remapped
   unsigned long long step_blocks; // blocks entering the first sweep of each acceleration step
};

__host__ __device__ inline void swapped_indices(uint32_t gid, const uint32_t len[3], int dim, uint32_t s[3]) {
   const uint32_t x = gid % len[0];
   const uint32_t y = (gid / len[0]) % len[1];
   const uint32_t z = gid / (len[0] * len[1]);
   if (dim == 0) { s[0] = z; s[1] = y; s[2] = x; }
   else if (dim == 1) { s[0] = x; s[1] = z; s[2] = y; }
   else { s[0] = x; s[1] = y; s[2] = z; }
}

__host__ __device__ inline uint32_t gid_from_swapped(uint32_t a, uint32_t b, uint32_t k, const uint32_t len[3], int dim) {
   uint32_t x, y, z;
   if (dim == 0) { z = a; y = b; x = k; }
   else if (dim == 1) { x = a; z = b; y = k; }
   else { x = a; y = b; z = k; }
   return x + len[0] * (y + len[1] * z);
}

// Transverse lengths (i, j) of the swapped frame.
__host__ __device__ inline void plane_lengths(const uint32_t len[3], int dim, uint32_t& li, uint32_t& lj) {
   if (dim == 0) { li = len[2]; lj = len[1]; }
   else if (dim == 1) { li = len[0]; lj = len[2]; }
   else { li = len[0]; lj = len[1]; }
}

__device__ inline int mask_popc_below(const uint32_t m[3], uint32_t k) {
   int n = 0;
   const uint32_t w = k >> 5, b = k & 31;
   if (w > 0) n += __popc(m[0]);
   if (w > 1) n += __popc(m[1]);
   n += __popc(m[w] & ((1u << b) - 1u));
   return n;
}

}  // namespace vlgpu
