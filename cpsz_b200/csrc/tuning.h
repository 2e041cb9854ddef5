// tuning.h -- launch-shape table of libcpsz_b200.
//
// Every parameter here changes how a kernel is launched (tile shape, threads
// per block, CTAs per SM, how a dimension is split, how many chunks an upload
// is cut into) and never what it computes: the bytes of every blob are the
// same for every value, which the GPU tests check for each parameter.
//
// The table maps (parameter, field size) to a value.  An entry applies to
// fields of at least `min_points` points; for a given size the entry with the
// largest such threshold wins, and a parameter without entries keeps its
// built-in default.  The offline sweep (cpsz_b200/autotune.py) measures each
// value per size bucket on the device and writes the table as JSON; the
// library loads it when the first context is created, from $CPSZ_B200_TUNING
// if set (empty or "none": no table), else from tuning_b200.json in the
// package directory (the parent of the library's directory) when present.
#pragma once

#include <cstdint>

#include <cstddef>

namespace cpsz {

enum TuneParam {
  TUNE_EB2D_TILE = 0,       // eb2d tile shape / threads (variant index, eb2d.cu)
  TUNE_WAVE2D_CTAS_PER_SM,  // resident wavefront CTAs per SM (0 = occupancy limit)
  TUNE_EB3D_FILL,           // eb3d: split i so the grid covers the SMs this many times
  TUNE_EB3D_MIN_CHUNK,      // eb3d: fewest i-planes one CTA marches over
  TUNE_H2D_CHUNKS,          // host-input uploads: row chunks overlapped with eb2d
  TUNE_WAVE2D_OVERLAP,      // 1: the wavefront runs beside eb2d (0: after it; tools
                            // that serialize kernels need 0, also set by
                            // the environment variable CPSZ_B200_OVERLAP=0)
  TUNE_EB2D_SKEW,           // beside the wavefront: eb2d's unit order, column
                            // blocks per group of lag (0: row order)
  TUNE_COUNT
};

struct TuneInfo {
  const char* name;
  int def, lo, hi;
};
const TuneInfo& tune_info(int p);
// Value of parameter p for a field (or pass) of `points` points.
int tune_get(TuneParam p, size_t points);
// Loads the default table once (no-op afterwards); returns a CPSZ status.
int tune_autoload();
// Changes with every change of the table (cached launch sequences key on it).
uint64_t tune_generation();

}  // namespace cpsz
