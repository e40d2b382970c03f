// Launch shapes of a batch's persistent kernels and the tuning table that
// picks them (no reference counterpart: the reference's GPU path uses fixed
// launch sizes).
//
// A batch runs its persistent kernels (the acceleration remap, the moments,
// the block adjustment, the translation walk) with a number of CTAs per SM.
// The default is each kernel's occupancy maximum; vlgpu_batch_set_launch sets
// others, and without such a call a batch consults the tuning table at every
// upload: the table (written by vlasiator_b200/autotune.py from timed steps)
// holds, per device name and bucket of mean blocks per cell, the shapes that
// were fastest.  Format, one entry per line, '#' starts a comment:
//
//   <device name>\t<lowest mean blocks per cell of the bucket>\t<remap>\t<moments>\t<adjust>\t<translate>
//
// The table is $VLGPU_LAUNCH_TABLE, else $XDG_CACHE_HOME/vlgpu/launch_table.tsv
// (~/.cache when XDG_CACHE_HOME is unset); a missing file means the defaults.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "batch_internal.cuh"

namespace vlgpu_batch_ops {

// Grid sizes from the requested shapes, each clamped to its kernel's
// occupancy maximum (the work arrays of the adjustment are sized for it).
void apply_launch(vlgpu_batch* b) {
   auto pick = [&](int k) {
      const int mx = b->cps_max[k] > 0 ? b->cps_max[k] : 1;
      const int want = (int)b->cps[k];
      return (want > 0 && want < mx) ? want : mx;
   };
   b->remap_grid = b->sm_count * pick(0);
   b->mom_grid = b->sm_count * pick(1);
   b->adj_grid = b->sm_count * pick(2);
}

std::string launch_table_path() {
   if (const char* p = std::getenv("VLGPU_LAUNCH_TABLE")) return p;
   std::string dir;
   if (const char* x = std::getenv("XDG_CACHE_HOME")) dir = x;
   else if (const char* h = std::getenv("HOME")) dir = std::string(h) + "/.cache";
   else return "";
   return dir + "/vlgpu/launch_table.tsv";
}

// The table's entry for the device and mean blocks per cell; false if none.
bool lookup_launch(const char* path, const char* device, double mean_blocks, vlgpu_launch* out) {
   if (!path || !*path || !device) return false;
   FILE* f = std::fopen(path, "r");
   if (!f) return false;
   char line[512];
   double best_min = -1.0;
   bool found = false;
   while (std::fgets(line, sizeof line, f)) {
      if (line[0] == '#' || line[0] == '\n') continue;
      char* tab = std::strchr(line, '\t');
      if (!tab) continue;
      *tab = '\0';
      if (std::strcmp(line, device) != 0) continue;
      double mn = 0.0;
      unsigned r = 0, m = 0, a = 0, t = 0;
      if (std::sscanf(tab + 1, "%lf\t%u\t%u\t%u\t%u", &mn, &r, &m, &a, &t) != 5) continue;
      if (mn <= mean_blocks && mn > best_min) {
         best_min = mn;
         out->remap_ctas_per_sm = r;
         out->moments_ctas_per_sm = m;
         out->adjust_ctas_per_sm = a;
         out->translate_ctas_per_sm = t;
         found = true;
      }
   }
   std::fclose(f);
   return found;
}

// At upload: the table's shapes for this device and the uploaded cells' mean
// block count, unless the caller set the shapes itself.
void consult_launch_table(vlgpu_batch* b, double mean_blocks) {
   if (b->launch_pinned) return;
   vlgpu_launch cfg{};
   const std::string path = launch_table_path();
   if (lookup_launch(path.c_str(), b->device_name, mean_blocks, &cfg)) {
      b->cps[0] = cfg.remap_ctas_per_sm;
      b->cps[1] = cfg.moments_ctas_per_sm;
      b->cps[2] = cfg.adjust_ctas_per_sm;
      b->cps[3] = cfg.translate_ctas_per_sm;
   } else {
      b->cps[0] = b->cps[1] = b->cps[2] = b->cps[3] = 0;
   }
   apply_launch(b);
}

}  // namespace vlgpu_batch_ops

using namespace vlgpu_batch_ops;

extern "C" {

int vlgpu_batch_set_launch(vlgpu_batch* b, const vlgpu_launch* cfg) {
   if (!b) return VLGPU_EINVAL;
   if (!cfg) {  // back to the table's (or the default) shapes at the next upload
      b->launch_pinned = false;
      b->cps[0] = b->cps[1] = b->cps[2] = b->cps[3] = 0;
   } else {
      b->launch_pinned = true;
      b->cps[0] = cfg->remap_ctas_per_sm;
      b->cps[1] = cfg->moments_ctas_per_sm;
      b->cps[2] = cfg->adjust_ctas_per_sm;
      b->cps[3] = cfg->translate_ctas_per_sm;
   }
   apply_launch(b);
   return VLGPU_OK;
}

int vlgpu_batch_get_launch(vlgpu_batch* b, vlgpu_launch* cfg) {
   if (!b || !cfg || b->sm_count <= 0) return VLGPU_EINVAL;
   cfg->remap_ctas_per_sm = (uint32_t)(b->remap_grid / b->sm_count);
   cfg->moments_ctas_per_sm = (uint32_t)(b->mom_grid / b->sm_count);
   cfg->adjust_ctas_per_sm = (uint32_t)(b->adj_grid / b->sm_count);
   cfg->translate_ctas_per_sm = b->cps[3];
   return VLGPU_OK;
}

int vlgpu_launch_table_lookup(const char* path, const char* device, double mean_blocks, vlgpu_launch* out) {
   if (!out || !device) return VLGPU_EINVAL;
   const std::string p = path ? std::string(path) : launch_table_path();
   return lookup_launch(p.c_str(), device, mean_blocks, out) ? VLGPU_OK : VLGPU_ENOENT;
}

}  // extern "C"
