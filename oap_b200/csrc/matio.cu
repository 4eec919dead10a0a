// Matrix files in the reference's format (layout in matio.cuh) and the
// C-ABI entry points that move them to and from device planes.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include "matio.cuh"
#include "oapb200.h"

namespace oapb {

namespace {

template <typename T>
void put(std::vector<char>& b, const T& v) {
  const char* p = reinterpret_cast<const char*>(&v);
  b.insert(b.end(), p, p + sizeof(T));
}

template <typename T>
bool get(const std::vector<char>& b, size_t& off, T* v) {
  if (off + sizeof(T) > b.size()) return false;
  memcpy(v, b.data() + off, sizeof(T));
  off += sizeof(T);
  return true;
}

}  // namespace

void matio_append(std::vector<char>& payload, const HostMat& m) {
  put<bool>(payload, m.present);
  if (!m.present) return;
  put<bool>(payload, m.has_re);
  put<bool>(payload, m.has_im);
  put<uint32_t>(payload, m.columns);
  put<uint32_t>(payload, m.rows);
  const size_t len = (size_t)m.columns * m.rows;
  if (m.has_re) {
    const char* p = reinterpret_cast<const char*>(m.re.data());
    payload.insert(payload.end(), p, p + sizeof(double) * len);
  }
  if (m.has_im) {
    const char* p = reinterpret_cast<const char*>(m.im.data());
    payload.insert(payload.end(), p, p + sizeof(double) * len);
  }
}

bool matio_parse(const std::vector<char>& payload, size_t& off, HostMat* out) {
  bool present = false;
  if (!get(payload, off, &present)) return false;
  out->present = present;
  if (!present) return true;
  if (!get(payload, off, &out->has_re) || !get(payload, off, &out->has_im) || !get(payload, off, &out->columns) ||
      !get(payload, off, &out->rows))
    return false;
  const size_t len = (size_t)out->columns * out->rows;
  for (int p = 0; p < 2; ++p) {
    const bool has = p == 0 ? out->has_re : out->has_im;
    std::vector<double>& v = p == 0 ? out->re : out->im;
    v.clear();
    if (!has) continue;
    if (off + sizeof(double) * len > payload.size()) return false;
    v.resize(len);
    memcpy(v.data(), payload.data() + off, sizeof(double) * len);
    off += sizeof(double) * len;
  }
  return true;
}

int matio_write_file(const char* path, const std::vector<char>& payload) {
  FILE* f = fopen(path, "wb");
  if (!f) return OAPB_ERR_ARG;
  const size_t elem = 1, len = payload.size();
  bool ok = fwrite(&elem, sizeof(size_t), 1, f) == 1 && fwrite(&len, sizeof(size_t), 1, f) == 1 &&
            (len == 0 || fwrite(payload.data(), 1, len, f) == len);
  ok = (fclose(f) == 0) && ok;
  return ok ? OAPB_OK : OAPB_ERR_ARG;
}

int matio_read_file(const char* path, std::vector<char>* payload) {
  FILE* f = fopen(path, "rb");
  if (!f) return OAPB_ERR_ARG;
  size_t elem = 0, len = 0;
  if (fread(&elem, sizeof(size_t), 1, f) != 1 || fread(&len, sizeof(size_t), 1, f) != 1 || elem != 1) {
    fclose(f);
    return OAPB_ERR_ARG;
  }
  // the header may announce more than the file holds (the reference writes
  // its allocated length): keep what is there
  payload->clear();
  char chunk[1 << 16];
  size_t got = 0;
  while (got < len) {
    const size_t want = len - got < sizeof(chunk) ? len - got : sizeof(chunk);
    const size_t r = fread(chunk, 1, want, f);
    if (r == 0) break;
    payload->insert(payload->end(), chunk, chunk + r);
    got += r;
  }
  fclose(f);
  return OAPB_OK;
}

}  // namespace oapb

using namespace oapb;

extern "C" {

int oapb_mat_write(const char* path, const oapb_mat* m, void* stream) {
  if (!path || !m || !m->re || m->dtype != OAPB_F64) return OAPB_ERR_ARG;
  HostMat h;
  h.columns = m->columns;
  h.rows = m->rows;
  h.has_re = true;
  h.has_im = m->im != nullptr;
  const size_t len = (size_t)m->columns * m->rows;
  cudaStream_t s = (cudaStream_t)stream;
  h.re.resize(len);
  if (cudaMemcpyAsync(h.re.data(), m->re, sizeof(double) * len, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return OAPB_ERR_CUDA;
  if (h.has_im) {
    h.im.resize(len);
    if (cudaMemcpyAsync(h.im.data(), m->im, sizeof(double) * len, cudaMemcpyDeviceToHost, s) != cudaSuccess)
      return OAPB_ERR_CUDA;
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return OAPB_ERR_CUDA;
  std::vector<char> payload;
  matio_append(payload, h);
  return matio_write_file(path, payload);
}

int oapb_mat_read_info(const char* path, uint32_t* columns, uint32_t* rows, int32_t* has_re, int32_t* has_im) {
  if (!path) return OAPB_ERR_ARG;
  std::vector<char> payload;
  int rc = matio_read_file(path, &payload);
  if (rc) return rc;
  size_t off = 0;
  HostMat h;
  if (!matio_parse(payload, off, &h) || !h.present) return OAPB_ERR_ARG;
  if (columns) *columns = h.columns;
  if (rows) *rows = h.rows;
  if (has_re) *has_re = h.has_re;
  if (has_im) *has_im = h.has_im;
  return OAPB_OK;
}

int oapb_mat_read(const char* path, const oapb_mat* dst, void* stream) {
  if (!path || !dst || !dst->re || dst->dtype != OAPB_F64) return OAPB_ERR_ARG;
  std::vector<char> payload;
  int rc = matio_read_file(path, &payload);
  if (rc) return rc;
  size_t off = 0;
  HostMat h;
  if (!matio_parse(payload, off, &h) || !h.present) return OAPB_ERR_ARG;
  if (h.columns != dst->columns || h.rows != dst->rows || (h.has_im && !dst->im)) return OAPB_ERR_ARG;
  const size_t len = (size_t)h.columns * h.rows;
  cudaStream_t s = (cudaStream_t)stream;
  if (h.has_re) {
    if (cudaMemcpyAsync(dst->re, h.re.data(), sizeof(double) * len, cudaMemcpyHostToDevice, s) != cudaSuccess)
      return OAPB_ERR_CUDA;
  } else if (cudaMemsetAsync(dst->re, 0, sizeof(double) * len, s) != cudaSuccess) {
    return OAPB_ERR_CUDA;
  }
  if (dst->im) {
    if (h.has_im) {
      if (cudaMemcpyAsync(dst->im, h.im.data(), sizeof(double) * len, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return OAPB_ERR_CUDA;
    } else if (cudaMemsetAsync(dst->im, 0, sizeof(double) * len, s) != cudaSuccess) {
      return OAPB_ERR_CUDA;
    }
  }
  return cudaStreamSynchronize(s) == cudaSuccess ? OAPB_OK : OAPB_ERR_CUDA;
}

}  // extern "C"
