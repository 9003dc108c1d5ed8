// Internal access to the storage of contiguous real(8) datasets of an open checkpoint file, so that
// the checkpoint transfers can move the data in parallel chunks (h5file.cpp; not part of the C ABI).
#pragma once
#include <cstdint>

#include "../../include/astr_b200.h"

namespace astr {

// Writes the object header of a real(8) dataset of Fortran shape dims (as astr_h5write_r8) and
// reserves its data; *fd, *offset: where the caller writes the n doubles (absolute file offset).
int h5_reserve_r8(astr_h5* h, const char* varname, int rank, const int64_t dims[], int* fd, uint64_t* offset);
// ASTR_OK with the file descriptor and absolute offset of the data when the dataset is stored
// contiguously as little-endian doubles with exactly the Fortran shape dims (mode 'h') or as a 1-D
// dataset of as many elements (mode 's'); ASTR_ERR_UNSUPPORTED otherwise (read it element-wise).
int h5_locate_r8(astr_h5* h, const char* varname, int rank, const int64_t dims[], char mode, int* fd,
                 uint64_t* offset);

}  // namespace astr
