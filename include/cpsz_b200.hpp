// cpsz_b200.hpp -- C++ drop-ins with the reference cpSZ signatures.
//
// libcpsz_b200.so exports these template instantiations (float and double)
// with the same mangled names as the reference's libcpsz, so a program built
// against the reference headers links against this library unchanged.  The
// float instantiations run the GPU path; the double ones return nullptr /
// leave the outputs null and set cpsz_b200_last_error() (the GPU kernels are
// written for float fields, the format of every workload here).
#ifndef CPSZ_B200_HPP
#define CPSZ_B200_HPP

#include <cstddef>

#include "cpsz_b200.h"

// include/sz_compress_cp_preserve_2d.hpp:10 (reference)
template <typename T>
unsigned char* sz_compress_cp_preserve_2d_offline(const T* U, const T* V, size_t r1, size_t r2,
                                                  size_t& compressed_size, bool transpose = false,
                                                  double max_pwr_eb = 0.1);

// include/sz_decompress_cp_preserve_2d.hpp:11 (reference)
template <typename T>
void sz_decompress_cp_preserve_2d_offline(const unsigned char* compressed, size_t r1, size_t r2, T*& U, T*& V);

// include/sz_compress_cp_preserve_2d.hpp:14 (reference)
template <typename T>
unsigned char* sz_compress_cp_preserve_2d_offline_log(const T* U, const T* V, size_t r1, size_t r2,
                                                      size_t& compressed_size, bool transpose = false,
                                                      double max_pwr_eb = 0.1);

// include/sz_decompress_cp_preserve_2d.hpp:15 (reference)
template <typename T>
void sz_decompress_cp_preserve_2d_offline_log(const unsigned char* compressed, size_t r1, size_t r2, T*& U, T*& V);

// include/sz_compress_cp_preserve_3d.hpp:8 (reference)
template <typename T>
unsigned char* sz_compress_cp_preserve_3d_offline_log(const T* U, const T* V, const T* W, size_t r1, size_t r2,
                                                      size_t r3, size_t& compressed_size, bool transpose = false,
                                                      double max_pwr_eb = 0.1);

// include/sz_decompress_cp_preserve_3d.hpp:11 (reference)
template <typename T>
void sz_decompress_cp_preserve_3d_online_log(const unsigned char* compressed, size_t r1, size_t r2, size_t r3, T*& U,
                                             T*& V, T*& W);

#endif
