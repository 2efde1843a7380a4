// checkpoint.cu -- exact binary checkpoints of a lattice.
//
// The reference's only way to resume is read_densities: it reloads the
// density field from a VTK file written with "%.4e" and starts the
// populations again from equilibrium (src/multiphase_lbm.cu:112-132), so a
// resumed run is not the run that was interrupted.  A checkpoint here holds
// the whole state in its stored precision: the populations of every node as
// the lattice keeps them (FP32, FP16 bits or FP64), the AA phase, the density
// field, the fluid mask and the parameters, plus the caller's step counter.
// Loading it into a lattice of the same size and storage and stepping on
// gives, bit for bit, what the uninterrupted lattice gives.
//
// Image layout (little-endian, host order): CkptHeader, then the mask words
// (lz * ly * wpr uint32), the density array (plane reals) and the
// populations (Q * plane elements), all in the lattice's internal dense
// layout (row pitch px).  A lattice held in the fluid-only layout is written
// through the dense layout (the conversion copies values, it rounds
// nothing).  payload_hash covers every byte after the header.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "capi_internal.h"
#include "kernels.cuh"

using namespace mlbm;

namespace {

constexpr char kMagic[8] = {'M', 'L', 'B', 'M', 'C', 'K', 'P', 'T'};
constexpr uint32_t kVersion = 1;

struct CkptHeader {
  char magic[8];
  uint32_t version;
  uint32_t header_bytes;
  int32_t lx, ly, lz, px;
  int32_t storage;
  int32_t phase;
  int64_t step;
  uint64_t mask_bytes, rho_bytes, pop_bytes;
  uint64_t payload_hash;
  mlbm_params params;
};

struct Sizes {
  uint64_t mask, rho, pop;
  uint64_t total() const { return sizeof(CkptHeader) + mask + rho + pop; }
};

Sizes sizes_of(const mlbm_lattice* lat) {
  const Geom& g = lat->g;
  Sizes s;
  s.mask = (uint64_t)g.lz * g.ly * g.wpr * sizeof(uint32_t);
  s.rho = (uint64_t)g.plane * real_bytes(lat->storage);
  s.pop = (uint64_t)g.plane * Q * pop_elem_bytes(lat->storage);
  return s;
}

// 64-bit FNV-1a over 8-byte words (the tail byte by byte): an integrity
// check of the image, not a cryptographic hash.
uint64_t image_hash(const unsigned char* p, uint64_t n) {
  uint64_t h = 0xcbf29ce484222325ull;
  const uint64_t prime = 0x100000001b3ull;
  uint64_t i = 0;
  for (; i + 8 <= n; i += 8) {
    uint64_t w;
    std::memcpy(&w, p + i, 8);
    h = (h ^ w) * prime;
  }
  for (; i < n; ++i) h = (h ^ p[i]) * prime;
  return h;
}

mlbm_status cuda_err(cudaError_t e, const char* where) {
  char msg[256];
  std::snprintf(msg, sizeof msg, "%s: %s", where, cudaGetErrorString(e));
  cudaGetLastError();
  return set_error(e == cudaErrorMemoryAllocation ? MLBM_ERR_NOMEM : MLBM_ERR_CUDA,
                   msg);
}

// psi of every node (ghost copies included) from the density array: the
// solid nodes' psi(rhos), which only initialisation writes otherwise.
template <typename R>
__global__ void k_psi_from_rho(const R* __restrict__ rho, R* __restrict__ psi,
                               Geom g, Phys p) {
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.lx || y >= g.ly) return;
  store_psi<R>(psi, g, x, y, z, psi_of<R>(p, rho[node_index(g, x, y, z)]));
}

mlbm_status check_header(const mlbm_lattice* lat, const CkptHeader& h,
                         uint64_t bytes) {
  const Sizes s = sizes_of(lat);
  if (std::memcmp(h.magic, kMagic, 8) != 0)
    return set_error(MLBM_ERR_ARG, "checkpoint: not a checkpoint image");
  if (h.version != kVersion || h.header_bytes != sizeof(CkptHeader))
    return set_error(MLBM_ERR_ARG, "checkpoint: unsupported format version");
  if (h.lx != lat->g.lx || h.ly != lat->g.ly || h.lz != lat->g.lz ||
      h.px != lat->g.px)
    return set_error(MLBM_ERR_ARG,
                     "checkpoint: lattice size differs from the image's");
  if (h.storage != lat->storage)
    return set_error(MLBM_ERR_ARG,
                     "checkpoint: population storage differs from the image's");
  if (h.mask_bytes != s.mask || h.rho_bytes != s.rho || h.pop_bytes != s.pop ||
      bytes < s.total())
    return set_error(MLBM_ERR_ARG, "checkpoint: image is truncated");
  if (h.phase != 0 && h.phase != 1)
    return set_error(MLBM_ERR_ARG, "checkpoint: invalid AA phase");
  return MLBM_OK;
}

}  // namespace

extern "C" {

mlbm_status mlbm_checkpoint_bytes(const mlbm_lattice* lat, uint64_t* bytes) {
  if (!lat || !bytes) return set_error(MLBM_ERR_ARG, "checkpoint: null argument");
  *bytes = sizes_of(lat).total();
  return MLBM_OK;
}

mlbm_status mlbm_checkpoint_info(const void* image, uint64_t bytes,
                                 int32_t* dims, int32_t* storage,
                                 int64_t* step) {
  if (!image) return set_error(MLBM_ERR_ARG, "checkpoint: null argument");
  if (bytes < sizeof(CkptHeader))
    return set_error(MLBM_ERR_ARG, "checkpoint: image is truncated");
  CkptHeader h;
  std::memcpy(&h, image, sizeof h);
  if (std::memcmp(h.magic, kMagic, 8) != 0)
    return set_error(MLBM_ERR_ARG, "checkpoint: not a checkpoint image");
  if (h.version != kVersion || h.header_bytes != sizeof(CkptHeader))
    return set_error(MLBM_ERR_ARG, "checkpoint: unsupported format version");
  if (dims) {
    dims[0] = h.lx;
    dims[1] = h.ly;
    dims[2] = h.lz;
  }
  if (storage) *storage = h.storage;
  if (step) *step = h.step;
  return MLBM_OK;
}

mlbm_status mlbm_checkpoint_save(mlbm_lattice* lat, int64_t step, void* image,
                                 uint64_t bytes) {
  if (!lat || !image) return set_error(MLBM_ERR_ARG, "checkpoint: null argument");
  if (!lat->initialized)
    return set_error(MLBM_ERR_STATE, "checkpoint: lattice not initialised");
  if (lat->slab)
    return set_error(MLBM_ERR_STATE,
                     "checkpoint: slab lattices are saved through their own "
                     "planes (gather them first)");
  const Sizes s = sizes_of(lat);
  if (bytes < s.total())
    return set_error(MLBM_ERR_ARG, "checkpoint: image buffer too small");
  DeviceGuard restore_device;
  cudaError_t e = cudaSetDevice(lat->device);
  if (e != cudaSuccess) return cuda_err(e, "checkpoint");
  // the fluid-only layout's values, copied into the dense buffer
  if (mlbm_status st = compact_sync_dense(lat)) return st;
  unsigned char* out = static_cast<unsigned char*>(image);
  unsigned char* payload = out + sizeof(CkptHeader);
  e = cudaMemcpyAsync(payload, lat->mask, s.mask, cudaMemcpyDefault, lat->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(payload + s.mask, lat->rho, s.rho, cudaMemcpyDefault,
                        lat->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(payload + s.mask + s.rho, lat->pop, s.pop,
                        cudaMemcpyDefault, lat->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(lat->stream);
  if (e != cudaSuccess) return cuda_err(e, "checkpoint save copy");
  CkptHeader h;
  std::memset(&h, 0, sizeof h);
  std::memcpy(h.magic, kMagic, 8);
  h.version = kVersion;
  h.header_bytes = sizeof(CkptHeader);
  h.lx = lat->g.lx;
  h.ly = lat->g.ly;
  h.lz = lat->g.lz;
  h.px = lat->g.px;
  h.storage = lat->storage;
  h.phase = lat->phase;
  h.step = step;
  h.mask_bytes = s.mask;
  h.rho_bytes = s.rho;
  h.pop_bytes = s.pop;
  h.params = lat->params;
  h.payload_hash = image_hash(payload, s.mask + s.rho + s.pop);
  std::memcpy(out, &h, sizeof h);
  return MLBM_OK;
}

mlbm_status mlbm_checkpoint_load(mlbm_lattice* lat, const void* image,
                                 uint64_t bytes, int64_t* step) {
  if (!lat || !image) return set_error(MLBM_ERR_ARG, "checkpoint: null argument");
  if (lat->slab)
    return set_error(MLBM_ERR_STATE, "checkpoint: cannot load into a slab lattice");
  if (bytes < sizeof(CkptHeader))
    return set_error(MLBM_ERR_ARG, "checkpoint: image is truncated");
  CkptHeader h;
  std::memcpy(&h, image, sizeof h);
  if (mlbm_status st = check_header(lat, h, bytes)) return st;
  const Sizes s = sizes_of(lat);
  const unsigned char* payload =
      static_cast<const unsigned char*>(image) + sizeof(CkptHeader);
  if (image_hash(payload, s.mask + s.rho + s.pop) != h.payload_hash)
    return set_error(MLBM_ERR_ARG, "checkpoint: image is corrupted (hash mismatch)");
  DeviceGuard restore_device;
  cudaError_t e = cudaSetDevice(lat->device);
  if (e != cudaSuccess) return cuda_err(e, "checkpoint");
  if (mlbm_status st = mlbm_set_params(lat, &h.params)) return st;
  e = cudaMemcpyAsync(lat->mask, payload, s.mask, cudaMemcpyDefault, lat->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(lat->rho, payload + s.mask, s.rho, cudaMemcpyDefault,
                        lat->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(lat->pop, payload + s.mask + s.rho, s.pop,
                        cudaMemcpyDefault, lat->stream);
  if (e != cudaSuccess) return cuda_err(e, "checkpoint load copy");
  const Geom& g = lat->g;
  const dim3 block(32, 4, 1), grid(g.px / 32, (g.ly + 3) / 4, g.lz);
  k_build_nbr<<<grid, block, 0, lat->stream>>>(lat->mask, lat->nbw, g, lat->phys);
  if (lat->storage == MLBM_STORE_F64)
    k_psi_from_rho<double><<<grid, block, 0, lat->stream>>>(
        static_cast<const double*>(lat->rho), static_cast<double*>(lat->psi), g,
        lat->phys);
  else
    k_psi_from_rho<float><<<grid, block, 0, lat->stream>>>(
        static_cast<const float*>(lat->rho), static_cast<float*>(lat->psi), g,
        lat->phys);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(lat->stream);
  if (e != cudaSuccess) return cuda_err(e, "checkpoint load");
  compact_invalidate(lat);  // the fluid-only tables follow the new mask
  lat->phase = h.phase;
  lat->has_mask = true;
  lat->has_rho = true;
  lat->initialized = true;
  lat->vel_valid = false;
  if (step) *step = h.step;
  return MLBM_OK;
}

mlbm_status mlbm_checkpoint_write(mlbm_lattice* lat, int64_t step,
                                  const char* path) {
  if (!lat || !path) return set_error(MLBM_ERR_ARG, "checkpoint: null argument");
  uint64_t bytes = 0;
  if (mlbm_status st = mlbm_checkpoint_bytes(lat, &bytes)) return st;
  std::vector<unsigned char> image;
  try {
    image.resize(bytes);
  } catch (...) {
    return set_error(MLBM_ERR_NOMEM, "checkpoint: host buffer");
  }
  if (mlbm_status st = mlbm_checkpoint_save(lat, step, image.data(), bytes))
    return st;
  FILE* f = std::fopen(path, "wb");
  if (!f) return set_error(MLBM_ERR_IO, "checkpoint: cannot open file for writing");
  const bool ok = std::fwrite(image.data(), 1, bytes, f) == bytes;
  if (std::fclose(f) != 0 || !ok)
    return set_error(MLBM_ERR_IO, "checkpoint: write failed");
  return MLBM_OK;
}

mlbm_status mlbm_checkpoint_read(mlbm_lattice* lat, const char* path,
                                 int64_t* step) {
  if (!lat || !path) return set_error(MLBM_ERR_ARG, "checkpoint: null argument");
  FILE* f = std::fopen(path, "rb");
  if (!f) return set_error(MLBM_ERR_IO, "checkpoint: cannot open file");
  long size = -1;
  if (std::fseek(f, 0, SEEK_END) == 0) size = std::ftell(f);
  if (size < 0 || std::fseek(f, 0, SEEK_SET) != 0) {
    std::fclose(f);
    return set_error(MLBM_ERR_IO, "checkpoint: cannot size file");
  }
  std::vector<unsigned char> image;
  try {
    image.resize((size_t)size);
  } catch (...) {
    std::fclose(f);
    return set_error(MLBM_ERR_NOMEM, "checkpoint: host buffer");
  }
  const bool ok = std::fread(image.data(), 1, image.size(), f) == image.size();
  std::fclose(f);
  if (!ok) return set_error(MLBM_ERR_IO, "checkpoint: read failed");
  return mlbm_checkpoint_load(lat, image.data(), image.size(), step);
}

}  // extern "C"
