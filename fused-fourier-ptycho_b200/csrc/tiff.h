// Host-side reader of the measured TIFF frames (one file per LED).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

namespace fpm {

enum class TiffOut {
    kU16,      // raw counts, single-sample images only
    kF32Mean,  // float mean over the samples of each pixel
};

// Reads the h x h pixel region whose top-left pixel is (row r0, column c0),
// 0-based, into page (column-major, h*h elements of the TiffOut type).
// Returns "" on success, else what is wrong with the file.
std::string read_tiff_region(const char *path, int r0, int c0, int h, TiffOut type, void *page);

// read_tiff_region over n files into consecutive pages of stack, on up to
// `threads` host threads (<= 0: one per hardware thread, at most 32).  On
// failure returns the message of the lowest-numbered failing file.
std::string read_tiff_stack(const char *const *paths, int n, int r0, int c0, int h, TiffOut type,
                            void *stack, int threads);

}  // namespace fpm
