// Checkpoint / pickup files in the logical layout of Write_Model2D and
// Read_Model2D (src/SELF_Model2D.f90:861-1099).  The reference writes HDF5
// groups (/quadrature, /state/interior, /state/boundary, /mesh/...) with the
// polynomial degree as attribute N; this container keeps the same dataset
// paths, Fortran-order shapes and attributes in a plain binary file, so a
// pickup needs no HDF5.
//
// File: "SELFCKP1", uint32 version, uint32 entry count, then entries
//   uint16 name length, name bytes, uint8 kind (0 array, 1 attribute),
//   uint8 dtype (1 f64, 2 i32, 3 f32), uint8 ndims, uint64 dims[ndims]
//   (first dimension fastest, as in Fortran), uint64 payload bytes, payload.
// All integers little-endian.  Arrays may come from device or host memory.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "selfgpu_internal.h"

using namespace selfgpu;

namespace {

const char kMagic[8] = {'S', 'E', 'L', 'F', 'C', 'K', 'P', '1'};
const uint32_t kVersion = 1;

size_t dtype_size(int dt) { return dt == SELFGPU_DT_F64 ? 8 : (dt == SELFGPU_DT_I32 || dt == SELFGPU_DT_F32) ? 4 : 0; }

struct Entry {
  int kind = 0, dtype = 0;
  std::vector<uint64_t> dims;
  uint64_t bytes = 0;
  long offset = 0;  // payload position
};

}  // namespace

struct selfgpu_ckpt {
  FILE* f = nullptr;
  bool write = false;
  uint32_t count = 0;
  long countPos = 0;
  std::map<std::string, Entry> index;
  std::vector<char> staging;
};

static int ckpt_fail(const std::string& msg) { return set_error(SELFGPU_ERR_ARG, msg); }

static bool put_bytes(FILE* f, const void* p, size_t n) { return fwrite(p, 1, n, f) == n; }
static bool get_bytes(FILE* f, void* p, size_t n) { return fread(p, 1, n, f) == n; }

extern "C" {

int selfgpu_ckpt_open(selfgpu_ckpt** out, const char* path, int write) {
  if (!out || !path) return ckpt_fail("selfgpu_ckpt_open: null argument");
  *out = nullptr;
  FILE* f = fopen(path, write ? "wb" : "rb");
  if (!f) return ckpt_fail(std::string("selfgpu_ckpt_open: cannot open ") + path);
  auto* c = new selfgpu_ckpt();
  c->f = f;
  c->write = write != 0;
  if (c->write) {
    uint32_t zero = 0;
    bool ok = put_bytes(f, kMagic, 8) && put_bytes(f, &kVersion, 4);
    c->countPos = ftell(f);
    ok = ok && put_bytes(f, &zero, 4);
    if (!ok) {
      fclose(f);
      delete c;
      return ckpt_fail("selfgpu_ckpt_open: write failed");
    }
  } else {
    char magic[8];
    uint32_t ver = 0, n = 0;
    if (!get_bytes(f, magic, 8) || std::memcmp(magic, kMagic, 8) != 0 || !get_bytes(f, &ver, 4) || ver != kVersion ||
        !get_bytes(f, &n, 4)) {
      fclose(f);
      delete c;
      return ckpt_fail(std::string("selfgpu_ckpt_open: not a checkpoint file: ") + path);
    }
    long fileSize = -1;
    const long here = ftell(f);
    if (fseek(f, 0, SEEK_END) == 0) fileSize = ftell(f);
    fseek(f, here, SEEK_SET);
    for (uint32_t k = 0; k < n; ++k) {
      uint16_t len = 0;
      uint8_t kind = 0, dt = 0, nd = 0;
      Entry en;
      std::string name;
      bool ok = get_bytes(f, &len, 2);
      if (ok) {
        name.resize(len);
        ok = get_bytes(f, &name[0], len) && get_bytes(f, &kind, 1) && get_bytes(f, &dt, 1) && get_bytes(f, &nd, 1);
      }
      if (ok && nd > 8) ok = false;
      if (ok) {
        en.dims.resize(nd);
        ok = (nd == 0 || get_bytes(f, en.dims.data(), 8 * (size_t)nd)) && get_bytes(f, &en.bytes, 8);
      }
      if (ok) {
        en.kind = kind;
        en.dtype = dt;
        en.offset = ftell(f);
        ok = fileSize >= 0 && (uint64_t)en.offset + en.bytes <= (uint64_t)fileSize &&
             fseek(f, (long)en.bytes, SEEK_CUR) == 0;
      }
      if (!ok) {
        fclose(f);
        delete c;
        return ckpt_fail(std::string("selfgpu_ckpt_open: truncated or corrupt checkpoint: ") + path);
      }
      c->index[name] = en;
    }
    c->count = n;
  }
  *out = c;
  return SELFGPU_OK;
}

static int ckpt_put_entry(selfgpu_ckpt* c, const char* name, int kind, int dtype, int ndims, const long long* dims,
                          const void* data, size_t bytes, int onDevice) {
  const size_t len = std::strlen(name);
  if (len == 0 || len > 65535) return ckpt_fail("selfgpu_ckpt_put: bad name");
  const void* src = data;
  if (onDevice && bytes) {
    c->staging.resize(bytes);
    cudaError_t e = cudaMemcpy(c->staging.data(), data, bytes, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return set_error(SELFGPU_ERR_CUDA, std::string("selfgpu_ckpt_put: ") + cudaGetErrorString(e));
    src = c->staging.data();
  }
  const uint16_t l16 = (uint16_t)len;
  const uint8_t k8 = (uint8_t)kind, d8 = (uint8_t)dtype, n8 = (uint8_t)ndims;
  std::vector<uint64_t> d64(ndims);
  for (int k = 0; k < ndims; ++k) d64[k] = (uint64_t)dims[k];
  const uint64_t b64 = bytes;
  bool ok = put_bytes(c->f, &l16, 2) && put_bytes(c->f, name, len) && put_bytes(c->f, &k8, 1) &&
            put_bytes(c->f, &d8, 1) && put_bytes(c->f, &n8, 1) &&
            (ndims == 0 || put_bytes(c->f, d64.data(), 8 * (size_t)ndims)) && put_bytes(c->f, &b64, 8) &&
            (bytes == 0 || put_bytes(c->f, src, bytes));
  if (!ok) return ckpt_fail("selfgpu_ckpt_put: write failed");
  ++c->count;
  return SELFGPU_OK;
}

int selfgpu_ckpt_put(selfgpu_ckpt* c, const char* name, const void* data, int dtype, int ndims, const long long* dims,
                     int onDevice) {
  if (!c || !c->write || !name || !data || ndims < 1 || ndims > 8 || !dims || !dtype_size(dtype))
    return ckpt_fail("selfgpu_ckpt_put: bad arguments");
  size_t n = 1;
  for (int k = 0; k < ndims; ++k) {
    if (dims[k] < 0) return ckpt_fail("selfgpu_ckpt_put: negative dimension");
    n *= (size_t)dims[k];
  }
  return ckpt_put_entry(c, name, 0, dtype, ndims, dims, data, n * dtype_size(dtype), onDevice);
}

int selfgpu_ckpt_put_attr(selfgpu_ckpt* c, const char* name, double value) {
  if (!c || !c->write || !name) return ckpt_fail("selfgpu_ckpt_put_attr: bad arguments");
  return ckpt_put_entry(c, name, 1, SELFGPU_DT_F64, 0, nullptr, &value, 8, 0);
}

int selfgpu_ckpt_info(selfgpu_ckpt* c, const char* name, int* dtype, int* ndims, long long* dims) {
  if (!c || c->write || !name) return ckpt_fail("selfgpu_ckpt_info: bad arguments");
  auto it = c->index.find(name);
  if (it == c->index.end()) return ckpt_fail(std::string("selfgpu_ckpt_info: no dataset ") + name);
  if (dtype) *dtype = it->second.dtype;
  if (ndims) *ndims = (int)it->second.dims.size();
  if (dims)
    for (size_t k = 0; k < it->second.dims.size(); ++k) dims[k] = (long long)it->second.dims[k];
  return SELFGPU_OK;
}

// Elements [elemOffset, elemOffset + nElem) of an array whose last dimension
// is the element index (a rank's slab, as Read_Model2D reads with MPI);
// elemOffset = 0, nElem = -1 reads the whole array.
int selfgpu_ckpt_get(selfgpu_ckpt* c, const char* name, void* data, long long capacityBytes, long long elemOffset,
                     long long nElem, int onDevice) {
  if (!c || c->write || !name || !data) return ckpt_fail("selfgpu_ckpt_get: bad arguments");
  auto it = c->index.find(name);
  if (it == c->index.end() || it->second.kind != 0) return ckpt_fail(std::string("selfgpu_ckpt_get: no array ") + name);
  const Entry& en = it->second;
  const uint64_t last = en.dims.empty() ? 1 : en.dims.back();
  const uint64_t per = last ? en.bytes / last : 0;
  if (nElem < 0) {
    elemOffset = 0;
    nElem = (long long)last;
  }
  if (elemOffset < 0 || (uint64_t)(elemOffset + nElem) > last)
    return ckpt_fail(std::string("selfgpu_ckpt_get: element range outside ") + name);
  const size_t bytes = (size_t)(per * (uint64_t)nElem);
  if ((long long)bytes > capacityBytes) return ckpt_fail(std::string("selfgpu_ckpt_get: buffer too small for ") + name);
  std::vector<char>& st = c->staging;
  char* dst = onDevice ? (st.resize(bytes), st.data()) : static_cast<char*>(data);
  if (fseek(c->f, en.offset + (long)(per * (uint64_t)elemOffset), SEEK_SET) != 0 || !get_bytes(c->f, dst, bytes))
    return ckpt_fail(std::string("selfgpu_ckpt_get: read failed for ") + name);
  if (onDevice && bytes) {
    cudaError_t e = cudaMemcpy(data, dst, bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return set_error(SELFGPU_ERR_CUDA, std::string("selfgpu_ckpt_get: ") + cudaGetErrorString(e));
  }
  return SELFGPU_OK;
}

int selfgpu_ckpt_get_attr(selfgpu_ckpt* c, const char* name, double* value) {
  if (!c || c->write || !name || !value) return ckpt_fail("selfgpu_ckpt_get_attr: bad arguments");
  auto it = c->index.find(name);
  if (it == c->index.end() || it->second.kind != 1)
    return ckpt_fail(std::string("selfgpu_ckpt_get_attr: no attribute ") + name);
  if (fseek(c->f, it->second.offset, SEEK_SET) != 0 || !get_bytes(c->f, value, 8))
    return ckpt_fail("selfgpu_ckpt_get_attr: read failed");
  return SELFGPU_OK;
}

int selfgpu_ckpt_close(selfgpu_ckpt* c) {
  if (!c) return SELFGPU_OK;
  bool ok = true;
  if (c->write) {
    ok = fseek(c->f, c->countPos, SEEK_SET) == 0 && put_bytes(c->f, &c->count, 4);
    ok = (fflush(c->f) == 0) && ok;
  }
  fclose(c->f);
  delete c;
  return ok ? SELFGPU_OK : ckpt_fail("selfgpu_ckpt_close: could not finalise the file");
}

// TimeStamp (src/SELF_SupportRoutines.f90:856-924), seconds: "DDDDHHMMSSmmm".
int selfgpu_time_stamp(double time, char* out) {
  if (!out) return ckpt_fail("selfgpu_time_stamp: null output");
  int day = (int)(time / 86400.0);
  int hour = (int)((time - 86400.0 * day) / 3600.0);
  int minute = (int)((time - 3600.0 * hour - 86400.0 * day) / 60.0);
  int second = (int)(time - 60.0 * minute - 3600.0 * hour - 86400.0 * day);
  // NINT: nearest integer, halves away from zero
  int ms = (int)std::lround(((time - 60.0 * minute - 3600.0 * hour - 86400.0 * day) - (double)second) * 1000.0);
  if (ms >= 1000) {
    ms -= 1000;
    second += 1;
  }
  if (second >= 60) {
    second -= 60;
    minute += 1;
  }
  if (minute >= 60) {
    minute -= 60;
    hour += 1;
  }
  if (hour >= 24) {
    hour -= 24;
    day += 1;
  }
  std::snprintf(out, 14, "%04d%02d%02d%02d%03d", day, hour, minute, second, ms);
  return SELFGPU_OK;
}

}  // extern "C"
