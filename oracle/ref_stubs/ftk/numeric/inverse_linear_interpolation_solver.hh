// Include-path stand-in for FTK's inverse-interpolation header.  The reference's
// 3D source includes it for its online_abs variant only (not on the offline
// path this oracle builds); the stub lets that translation unit compile and is
// never called by the offline_log compressor or the online_log decoder.
#pragma once
#include <cstdlib>
namespace ftk {
template <typename T>
inline bool inverse_lerp_s3v3(const T[4][3], double mu[4], double* cond, double threshold = 0.0) {
  (void)mu; (void)cond; (void)threshold;
  std::abort();  // unreachable from the offline path
  return false;
}
}  // namespace ftk
