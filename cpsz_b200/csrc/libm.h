// libm.h -- reproducing the host C library's single-precision log2f / exp2f
// on the GPU, bit for bit.
//
// The reference's 3D path applies log2f to every field value
// (include/sz_cp_preserve_utils.hpp:201-216) and exp2f to every decoded log
// value (src/sz_decompress_cp_preserve_3d.cpp:95-104).  glibc's versions are
// not correctly rounded, so a GPU that rounded the exact result would differ
// on a few hundred thousand inputs.  The library therefore scans every float
// input of both functions once (all positive floats for log2f, [-99, 128] for
// exp2f), with 64-bit-mantissa long double as the exact reference, and keeps
//   hard  inputs whose exact result lies within 2^-18 ulp of a rounding
//         midpoint, with the host library's output;
//   mis   the other inputs where the host library returned the neighbour on
//         the far side of the midpoint, and per input binade (sign and
//         exponent of the input) the largest midpoint distance among them.
// On the GPU a double-precision log2 / exp2 (error far below 2^-27 float ulp)
// then identifies the correctly rounded float and its midpoint distance d:
//   d < 2^-18 + margin      -> look the input up in `hard`;
//   d <= band(binade)+margin -> flip to the far neighbour if the input is in
//                              `mis` (a bitmap for the binades near 1, where
//                              glibc's log2f misrounds by up to 0.25 ulp);
//   otherwise               -> the correctly rounded float is glibc's answer.
// The scan takes about a minute on 8 cores; its result is cached in a file
// beside the shared library (regenerated when the C library version differs).
#pragma once

#include <cstdint>

struct cpsz_b200_ctx;

namespace cpsz {

// Device view of one function's tables.  Keys are input bits >> 23.
struct LibmFn {
  const uint32_t* hard_in;   // sorted input bits
  const uint32_t* hard_out;  // host library output bits
  const uint32_t* hard_off;  // 513 offsets into hard_* by key
  const uint32_t* mis;       // sorted input bits
  const uint32_t* mis_off;   // 513 offsets into mis by key
  const double* band;        // 512: largest misround distance per key (+ margin), -1 when none
  const int* bmp_slot;       // 512: bitmap slot per key or -1
  const uint32_t* bmp;       // slot s: 2^18 words, bit m = mantissa m misrounds
};
struct LibmTables {
  LibmFn log2f, exp2f;
};

// Uploads the tables to the context's device once (generating or loading the
// cache file on first use) and returns the device view.
int libm_tables_device(cpsz_b200_ctx* ctx, LibmTables* out);

// Loads (or generates and caches at `path`, or the default path when null)
// the host tables; returns CPSZ_OK or an error code with the last error set.
int libm_tables_prepare(const char* path);

}  // namespace cpsz
