// The reference's matrix file format, host side.
//
// A file is one utils::ByteBuffer over char (oapUtils/Buffer.h:207-270):
//   size_t element size (1) | size_t length | `length` payload bytes
// (the reference writes its allocated length and the used bytes; a reader
// takes what the file holds).  The payload is a sequence of matrices, each
// as oap::host::SaveMatrix writes it (oapMatrixCpu/oapHostMatrixUtils.cpp:
// 1054-1080, LoadMatrix / LoadMatrixInfo :1082-1113), packed, with the
// reference's build types (uintt = 32-bit, floatt = double):
//   bool present | bool isRe | bool isIm | uint32 columns | uint32 rows |
//   re[columns * rows] | im[columns * rows]       (row-major, (c, r) at c + r columns)
#pragma once

#include <stddef.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace oapb {

struct HostMat {
  bool present = true;
  bool has_re = true, has_im = false;
  uint32_t columns = 0, rows = 0;
  std::vector<double> re, im;
};

void matio_append(std::vector<char>& payload, const HostMat& m);
// parse the matrix at `off` (advanced past it); false when the payload is short
bool matio_parse(const std::vector<char>& payload, size_t& off, HostMat* out);
int matio_write_file(const char* path, const std::vector<char>& payload);
int matio_read_file(const char* path, std::vector<char>* payload);

}  // namespace oapb
