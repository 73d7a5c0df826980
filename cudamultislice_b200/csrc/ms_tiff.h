// ms_tiff.h -- float32 TIFF output (see ms_tiff.cu).
#pragma once

namespace ms {
// Writes nx x ny floats (row-major, row 0 at the top) to `path`.
// Returns 0 on success, 1 for bad arguments, 2 for an I/O failure.
int write_tiff_f32(const char* path, const float* data, int nx, int ny);
}  // namespace ms
