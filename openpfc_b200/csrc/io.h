// io.h -- on-disk formats of the reference's writers and readers, host side.
//
//  * File names: pfc::utils::format_with_number (frontend/utils/utils.hpp:96-139):
//    a pattern with no '%' is used as is; otherwise it must hold exactly one
//    printf integer conversion %d with optional flags "-+ 0", an optional '*'
//    and an optional width, and nothing else with a '%'.
//  * Raw binary (BinaryWriter / BinaryReader, frontend/io/binary_writer.hpp,
//    kernel/simulation/binary_reader.hpp): the global array as native doubles
//    (complex: re, im pairs), x fastest (MPI_ORDER_FORTRAN subarray of the
//    global box), no header; a writer truncates the file first.
//  * VTK XML ImageData (VTKWriter, src/openpfc/frontend/io/vtk_writer.cpp:70-108):
//    one Float64 point array, appended raw, header_type UInt64 length prefix,
//    numbers in the iostream default format (%g).
#pragma once
#include <stddef.h>

#include <string>

namespace opfc {
namespace io {

// OPFC_OK, or OPFC_ERR_ARG with a message for an invalid pattern.
int format_with_number(const char *pattern, int increment, std::string &out, std::string &err);

// Write / read `count` doubles of the box `local` at `offset` of the global
// array `global` (x fastest).  OPFC_ERR_IO on a file error, OPFC_ERR_SIZE when a
// read finds fewer bytes than the box needs.  A write of the whole array
// truncates the file first; a smaller box is written in place (the file is
// created if missing, never truncated), so several writers can fill one file.
int write_box(const std::string &fn, const int global[3], const int local[3], const int offset[3],
              const double *data, int ncomp, std::string &err);
// Truncate `fn` and size it to the whole global array (zeros): done once by a
// coordinator before several writers each write their box.
int prepare_box_file(const std::string &fn, const int global[3], int ncomp, std::string &err);
int read_box(const std::string &fn, const int global[3], const int local[3], const int offset[3], double *data,
             int ncomp, std::string &err);

// One .vti file for a piece `local` at `offset` of the global box.
int write_vti(const std::string &fn, const int global[3], const int local[3], const int offset[3],
              const double origin[3], const double spacing[3], const char *name, const double *data,
              std::string &err);

}  // namespace io
}  // namespace opfc
