// batch.cu -- host side of include/mlbm_batch.h: domain table, work lists,
// persistent batched launches, CUDA graph replay, autotuner.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <new>
#include <type_traits>
#include <vector>

#include "../../include/mlbm_batch.h"
#include "batch.cuh"
#include "batch_compact.cuh"
#include "capi_internal.h"

using namespace mlbm;

struct mlbm_batch {
  int storage = MLBM_STORE_F32;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<mlbm_lattice*> dom;     // slots (nullptr = free)
  std::vector<long long> origin;      // batch step at which step 0 would be
  std::vector<int> phase_base;        // AA phase offset (see DomainDesc)
  long long bstep = 0;                // steps executed by the batch
  // device tables, rebuilt when the set of domains or the tuning changes
  DomainDesc* d_desc = nullptr;
  long long* d_pre_d = nullptr;
  long long* d_pre_u = nullptr;
  long long* d_step = nullptr;
  int cap = 0;
  int nactive = 0;
  bool dirty = true;
  // tuning
  int By_d = 4, By_u = 4, Dz = 8, bps = 0, use_graphs = 1;
  int grid_d = 0, grid_u = 0;
  // graph of kGraphSteps steps (no rho output), for the current tables
  cudaGraphExec_t graph = nullptr;
  // compact mode (FP32 / FP16 storage, every domain within the compact
  // kernels' limits): the domains live in the fluid-only layout and every
  // pass is one launch over all of them (batch_compact.cuh)
  bool compact = false;
  CDomain* d_cdesc = nullptr;
  // block prefixes: [2][n + 1] of the density pass per step parity, then
  // [n + 1] of the update pass (node pairs in both AA phases)
  long long* d_cpre = nullptr;
  int ccap = 0;
  int grid_c = 0, grid_cu = 0;
};

namespace {

constexpr int kGraphSteps = 8;

__global__ void k_advance_step(long long* step, int n) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *step += n;
}

mlbm_status bfail(mlbm_status st, const char* msg) { return set_error(st, msg); }

#define BCUDA(expr, where)                                   \
  do {                                                       \
    cudaError_t _e = (expr);                                 \
    if (_e != cudaSuccess) return cuda_fail(_e, where);      \
  } while (0)

void drop_graph(mlbm_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
}

template <typename T>
const void* density_fn() { return reinterpret_cast<const void*>(&k_batch_density<T>); }
template <typename T>
const void* update_fn() { return reinterpret_cast<const void*>(&k_batch_update<T>); }

const void* pick_density(int storage) {
  return storage == MLBM_STORE_F32   ? density_fn<float>()
         : storage == MLBM_STORE_F16 ? density_fn<__half>()
                                     : density_fn<double>();
}
const void* pick_update(int storage) {
  return storage == MLBM_STORE_F32   ? update_fn<float>()
         : storage == MLBM_STORE_F16 ? update_fn<__half>()
                                     : update_fn<double>();
}

// Compact mode: every domain enters the fluid-only layout; block prefixes
// of the density pass for both step parities (one node per thread in the
// gather step, one pair per thread in the local step) and of the update
// pass (one pair per thread in both).
mlbm_status rebuild_compact(mlbm_batch* b) {
  std::vector<CDomain> desc;
  std::vector<long long> pre[2] = {std::vector<long long>(1, 0),
                                   std::vector<long long>(1, 0)};
  std::vector<long long> upre(1, 0);
  for (size_t s = 0; s < b->dom.size(); ++s) {
    mlbm_lattice* lat = b->dom[s];
    if (!lat) continue;
    if (mlbm_status st = compact_enter(lat)) return st;
    const CompactState& c = lat->compact;
    CDomain d;
    std::memset(&d, 0, sizeof d);
    d.g = lat->g;
    d.p = lat->phys;
    d.cpop = c.cpop;
    d.cinfo = c.cinfo;
    d.wtab = c.wtab;
    d.psi = static_cast<float*>(lat->psi);
    d.rho = static_cast<float*>(lat->rho);
    d.cs = (uint32_t)c.cs;
    d.nfluid = (int)c.nfluid;
    d.phase_base = b->phase_base[s];
    d.step_origin = b->origin[s];
    desc.push_back(d);
    for (int par = 0; par < 2; ++par) {
      const int ph = d.phase_base ^ par;
      const long long threads = ph == 0 ? d.nfluid : d.nfluid / 2;
      pre[par].push_back(pre[par].back() + (threads + kBCThreads - 1) / kBCThreads);
    }
    upre.push_back(upre.back() + (d.nfluid / 2 + kBCThreads - 1) / kBCThreads);
  }
  const int n = (int)desc.size();
  if (n > kMaxBatch) return bfail(MLBM_ERR_ARG, "too many domains in a batch");
  if (n > b->ccap) {
    cudaFree(b->d_cdesc);
    cudaFree(b->d_cpre);
    b->d_cdesc = nullptr;
    b->d_cpre = nullptr;
    const int cap = std::max(n, 64);
    BCUDA(cudaMalloc(&b->d_cdesc, cap * sizeof(CDomain)), "batch table");
    BCUDA(cudaMalloc(&b->d_cpre, 3 * (cap + 1) * sizeof(long long)), "batch table");
    b->ccap = cap;
  }
  std::vector<long long> both(pre[0]);
  both.insert(both.end(), pre[1].begin(), pre[1].end());
  both.insert(both.end(), upre.begin(), upre.end());
  if (n)
    BCUDA(cudaMemcpyAsync(b->d_cdesc, desc.data(), n * sizeof(CDomain),
                          cudaMemcpyHostToDevice, b->stream), "batch table");
  BCUDA(cudaMemcpyAsync(b->d_cpre, both.data(), both.size() * sizeof(long long),
                        cudaMemcpyHostToDevice, b->stream), "batch table");
  BCUDA(cudaMemcpyAsync(b->d_step, &b->bstep, sizeof(long long),
                        cudaMemcpyHostToDevice, b->stream), "batch step");
  BCUDA(cudaStreamSynchronize(b->stream), "batch table");
  b->nactive = n;
  b->grid_c = (int)std::max<long long>(1, std::max(pre[0].back(), pre[1].back()));
  b->grid_cu = (int)std::max<long long>(1, upre.back());
  b->dirty = false;
  return MLBM_OK;
}

bool compact_mode(const mlbm_batch* b) {
  if (b->storage == MLBM_STORE_F64) return false;
  for (mlbm_lattice* lat : b->dom)
    if (lat && !lat->compact.two_pass_ok) return false;
  return true;
}

mlbm_status rebuild(mlbm_batch* b) {
  drop_graph(b);
  b->compact = compact_mode(b);
  if (b->compact) return rebuild_compact(b);
  // dense mode: the domains stay on (or return to) the dense layout
  for (mlbm_lattice* lat : b->dom)
    if (lat)
      if (mlbm_status st = compact_leave(lat)) return st;
  std::vector<DomainDesc> desc;
  std::vector<long long> pre_d(1, 0), pre_u(1, 0);
  for (size_t s = 0; s < b->dom.size(); ++s) {
    mlbm_lattice* lat = b->dom[s];
    if (!lat) continue;
    DomainDesc d;
    std::memset(&d, 0, sizeof d);
    d.g = lat->g;
    d.p = lat->phys;
    d.pop = lat->pop;
    d.nbw = lat->nbw;
    d.psi = lat->psi;
    d.rho = lat->rho;
    d.vel = lat->vel;
    d.phase_base = b->phase_base[s];
    d.step_origin = b->origin[s];
    d.ntx = d.g.px / 32;
    d.nty_d = (d.g.ly + b->By_d - 1) / b->By_d;
    d.nty_u = (d.g.ly + b->By_u - 1) / b->By_u;
    d.nzc = (d.g.lz + b->Dz - 1) / b->Dz;
    desc.push_back(d);
    pre_d.push_back(pre_d.back() + (long long)d.ntx * d.nty_d * d.g.lz);
    pre_u.push_back(pre_u.back() + (long long)d.ntx * d.nty_u * d.nzc);
  }
  const int n = (int)desc.size();
  if (n > kMaxBatch) return bfail(MLBM_ERR_ARG, "too many domains in a batch");
  if (n > b->cap) {
    cudaFree(b->d_desc);
    cudaFree(b->d_pre_d);
    cudaFree(b->d_pre_u);
    b->d_desc = nullptr;
    b->d_pre_d = b->d_pre_u = nullptr;
    const int cap = std::max(n, 64);
    BCUDA(cudaMalloc(&b->d_desc, cap * sizeof(DomainDesc)), "batch table");
    BCUDA(cudaMalloc(&b->d_pre_d, (cap + 1) * sizeof(long long)), "batch table");
    BCUDA(cudaMalloc(&b->d_pre_u, (cap + 1) * sizeof(long long)), "batch table");
    b->cap = cap;
  }
  if (n) {
    BCUDA(cudaMemcpyAsync(b->d_desc, desc.data(), n * sizeof(DomainDesc),
                          cudaMemcpyHostToDevice, b->stream), "batch table");
  }
  BCUDA(cudaMemcpyAsync(b->d_pre_d, pre_d.data(), (n + 1) * sizeof(long long),
                        cudaMemcpyHostToDevice, b->stream), "batch table");
  BCUDA(cudaMemcpyAsync(b->d_pre_u, pre_u.data(), (n + 1) * sizeof(long long),
                        cudaMemcpyHostToDevice, b->stream), "batch table");
  BCUDA(cudaMemcpyAsync(b->d_step, &b->bstep, sizeof(long long),
                        cudaMemcpyHostToDevice, b->stream), "batch step");
  BCUDA(cudaStreamSynchronize(b->stream), "batch table");
  b->nactive = n;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device);
  int per_d = 0, per_u = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_d, pick_density(b->storage),
                                                32 * b->By_d, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_u, pick_update(b->storage),
                                                32 * b->By_u, 0);
  if (b->bps > 0) {
    per_d = std::min(per_d, b->bps);
    per_u = std::min(per_u, b->bps);
  }
  b->grid_d = (int)std::max<long long>(
      1, std::min<long long>((long long)std::max(per_d, 1) * nsm, pre_d.back()));
  b->grid_u = (int)std::max<long long>(
      1, std::min<long long>((long long)std::max(per_u, 1) * nsm, pre_u.back()));
  b->dirty = false;
  return MLBM_OK;
}

template <typename T>
void launch_step(mlbm_batch* b, int delta, int reverse, unsigned inject,
                 bool write_rho) {
  if constexpr (!std::is_same<T, double>::value) {
    if (b->compact) {
      if (write_rho)
        k_batch_cdensity<T, true><<<b->grid_c, kBCThreads, 0, b->stream>>>(
            b->d_cdesc, b->d_cpre, b->nactive, b->d_step, delta, reverse, inject);
      else
        k_batch_cdensity<T, false><<<b->grid_c, kBCThreads, 0, b->stream>>>(
            b->d_cdesc, b->d_cpre, b->nactive, b->d_step, delta, reverse, inject);
      k_batch_cupdate<T><<<b->grid_cu, kBCThreads, 0, b->stream>>>(
          b->d_cdesc, b->d_cpre + 2 * (b->nactive + 1), b->nactive, b->d_step,
          delta, reverse, inject);
      return;
    }
  }
  BatchArgs a;
  a.ndomains = b->nactive;
  a.By_d = b->By_d;
  a.By_u = b->By_u;
  a.Dz = b->Dz;
  a.reverse = reverse;
  a.inject_type = inject;
  a.write_rho = write_rho ? 1 : 0;
  k_batch_density<T><<<b->grid_d, 32 * b->By_d, 0, b->stream>>>(
      b->d_desc, b->d_pre_d, b->d_step, delta, a);
  k_batch_update<T><<<b->grid_u, 32 * b->By_u, 0, b->stream>>>(
      b->d_desc, b->d_pre_u, b->d_step, delta, a);
}

void launch_step_any(mlbm_batch* b, int delta, int reverse, unsigned inject,
                     bool write_rho) {
  if (b->storage == MLBM_STORE_F32)
    launch_step<float>(b, delta, reverse, inject, write_rho);
  else if (b->storage == MLBM_STORE_F16)
    launch_step<__half>(b, delta, reverse, inject, write_rho);
  else
    launch_step<double>(b, delta, reverse, inject, write_rho);
}

// Run n steps: the first n-1 without rho output (graph replays of
// kGraphSteps steps where possible), the last one writing rho.
mlbm_status run_steps(mlbm_batch* b, int n, int reverse, unsigned inject) {
  int done = 0;
  if (b->use_graphs && (reverse != 1 || inject != 0)) {
    // graphs are captured for the default injection arguments only
  } else if (b->use_graphs) {
    while (n - 1 - done >= kGraphSteps) {
      if (!b->graph) {
        cudaGraph_t g = nullptr;
        BCUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal),
              "graph capture");
        for (int j = 0; j < kGraphSteps; ++j)
          launch_step_any(b, j, reverse, inject, false);
        k_advance_step<<<1, 32, 0, b->stream>>>(b->d_step, kGraphSteps);
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (e != cudaSuccess) return cuda_fail(e, "graph capture");
        e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(e, "graph instantiate");
      }
      BCUDA(cudaGraphLaunch(b->graph, b->stream), "graph launch");
      done += kGraphSteps;
    }
  }
  for (; done < n; ++done) {
    launch_step_any(b, 0, reverse, inject, done == n - 1);
    k_advance_step<<<1, 32, 0, b->stream>>>(b->d_step, 1);
  }
  BCUDA(cudaGetLastError(), "batch launch");
  return MLBM_OK;
}

}  // namespace

namespace {
// Put an initialised (or restored) lattice into a free slot; it joins at the
// next iterate call with its step counter at step0.
int32_t insert_domain(mlbm_batch* b, mlbm_lattice* lat, int64_t step0) {
  int slot = -1;
  for (size_t s = 0; s < b->dom.size(); ++s)
    if (!b->dom[s]) { slot = (int)s; break; }
  if (slot < 0) {
    slot = (int)b->dom.size();
    b->dom.push_back(nullptr);
    b->origin.push_back(0);
    b->phase_base.push_back(0);
  }
  b->dom[slot] = lat;
  b->origin[slot] = b->bstep - step0;
  b->phase_base[slot] = (lat->phase + (int)(b->bstep & 1)) & 1;
  b->dirty = true;
  return slot;
}
}  // namespace

extern "C" {

mlbm_status mlbm_batch_create(int32_t storage, int32_t device,
                              mlbm_batch** out) {
  if (!out) return bfail(MLBM_ERR_ARG, "null output");
  *out = nullptr;
  if (storage < MLBM_STORE_F32 || storage > MLBM_STORE_F64)
    return bfail(MLBM_ERR_ARG, "invalid storage");
  int ndev = 0;
  BCUDA(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
  if (device < 0 || device >= ndev) return bfail(MLBM_ERR_CUDA, "device not available");
  mlbm::DeviceGuard restore_device;
  BCUDA(cudaSetDevice(device), "cudaSetDevice");
  mlbm_batch* b = new (std::nothrow) mlbm_batch();
  if (!b) return bfail(MLBM_ERR_NOMEM, "host allocation");
  b->storage = storage;
  b->device = device;
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_step, sizeof(long long));
  if (e != cudaSuccess) {
    mlbm_batch_destroy(b);
    return cuda_fail(e, "batch creation");
  }
  *out = b;
  return MLBM_OK;
}

mlbm_status mlbm_batch_destroy(mlbm_batch* b) {
  if (!b) return MLBM_OK;
  mlbm::DeviceGuard restore_device;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graph(b);
  for (mlbm_lattice* lat : b->dom)
    if (lat) mlbm_lattice_destroy(lat);
  cudaFree(b->d_cdesc);
  cudaFree(b->d_cpre);
  cudaFree(b->d_desc);
  cudaFree(b->d_pre_d);
  cudaFree(b->d_pre_u);
  cudaFree(b->d_step);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return MLBM_OK;
}

mlbm_status mlbm_batch_add(mlbm_batch* b, int32_t nx, int32_t ny, int32_t nz,
                           const mlbm_params* params, const uint8_t* is_fluid,
                           const float* rho, int64_t step0, int32_t* id) {
  if (!b || !params || !is_fluid || !rho || !id)
    return bfail(MLBM_ERR_ARG, "null argument");
  mlbm::DeviceGuard restore_device;
  BCUDA(cudaSetDevice(b->device), "cudaSetDevice");
  mlbm_lattice* lat = nullptr;
  if (mlbm_status st = mlbm_lattice_create(nx, ny, nz, b->storage, b->device, &lat))
    return st;
  // a domain advanced on its own (mlbm_iterate on its lattice) uses the
  // kernels bit-identical to the batch's: the compact two-pass step where the
  // compact kernels fit, else the dense two-pass step
  mlbm_status st = mlbm_set_stream(lat, b->stream);
  if (!st)
    st = mlbm_set_step_kernel(lat, lat->compact.two_pass_ok ? MLBM_KERNEL_COMPACT
                                                           : MLBM_KERNEL_TWO_PASS);
  if (!st) st = mlbm_set_params(lat, params);
  if (!st) st = mlbm_upload_fluid_mask(lat, is_fluid);
  if (!st) st = mlbm_upload_rho(lat, rho);
  if (!st) st = mlbm_initialize(lat);
  if (st) {
    mlbm_lattice_destroy(lat);
    return st;
  }
  *id = insert_domain(b, lat, step0);
  return MLBM_OK;
}

mlbm_status mlbm_batch_add_checkpoint(mlbm_batch* b, const void* image,
                                      uint64_t bytes, int32_t* id) {
  if (!b || !image || !id) return bfail(MLBM_ERR_ARG, "null argument");
  int32_t dims[3], storage;
  int64_t step0 = 0;
  if (mlbm_status st = mlbm_checkpoint_info(image, bytes, dims, &storage, &step0))
    return st;
  if (storage != b->storage)
    return bfail(MLBM_ERR_ARG, "checkpoint storage differs from the batch's");
  mlbm::DeviceGuard restore_device;
  BCUDA(cudaSetDevice(b->device), "cudaSetDevice");
  mlbm_lattice* lat = nullptr;
  if (mlbm_status st = mlbm_lattice_create(dims[0], dims[1], dims[2], b->storage,
                                           b->device, &lat))
    return st;
  mlbm_status st = mlbm_set_stream(lat, b->stream);
  if (!st)
    st = mlbm_set_step_kernel(lat, lat->compact.two_pass_ok ? MLBM_KERNEL_COMPACT
                                                           : MLBM_KERNEL_TWO_PASS);
  if (!st) st = mlbm_checkpoint_load(lat, image, bytes, &step0);
  if (st) {
    mlbm_lattice_destroy(lat);
    return st;
  }
  *id = insert_domain(b, lat, step0);
  return MLBM_OK;
}


mlbm_status mlbm_batch_remove(mlbm_batch* b, int32_t id) {
  if (!b || id < 0 || id >= (int)b->dom.size() || !b->dom[id])
    return bfail(MLBM_ERR_ARG, "no such domain");
  BCUDA(cudaStreamSynchronize(b->stream), "batch remove");
  mlbm_lattice_destroy(b->dom[id]);
  b->dom[id] = nullptr;
  b->dirty = true;
  return MLBM_OK;
}

int32_t mlbm_batch_count(const mlbm_batch* b) {
  if (!b) return 0;
  int n = 0;
  for (mlbm_lattice* l : b->dom) n += l ? 1 : 0;
  return n;
}

uint64_t mlbm_batch_bytes(const mlbm_batch* b) {
  if (!b) return 0;
  uint64_t s = 0;
  for (mlbm_lattice* l : b->dom)
    if (l) s += mlbm_lattice_bytes(l->g.lx, l->g.ly, l->g.lz, b->storage);
  return s;
}

mlbm_status mlbm_batch_iterate(mlbm_batch* b, int32_t nsteps, int32_t reverse,
                               uint32_t inject_type) {
  if (!b) return bfail(MLBM_ERR_ARG, "null batch");
  if (nsteps < 0) return bfail(MLBM_ERR_ARG, "negative step count");
  if (nsteps == 0) return MLBM_OK;
  mlbm::DeviceGuard restore_device;
  BCUDA(cudaSetDevice(b->device), "cudaSetDevice");
  if (b->dirty)
    if (mlbm_status st = rebuild(b)) return st;
  if (b->nactive == 0) return MLBM_OK;
  if (mlbm_status st = run_steps(b, nsteps, reverse, inject_type)) return st;
  b->bstep += nsteps;
  for (mlbm_lattice* l : b->dom)
    if (l) {
      l->phase = (l->phase + nsteps) & 1;
    }
  return MLBM_OK;
}

mlbm_lattice* mlbm_batch_lattice(mlbm_batch* b, int32_t id) {
  if (!b || id < 0 || id >= (int)b->dom.size()) return nullptr;
  return b->dom[id];
}

int64_t mlbm_batch_domain_step(const mlbm_batch* b, int32_t id) {
  if (!b || id < 0 || id >= (int)b->dom.size() || !b->dom[id]) return -1;
  return b->bstep - b->origin[id];
}

mlbm_status mlbm_batch_synchronize(mlbm_batch* b) {
  if (!b) return bfail(MLBM_ERR_ARG, "null batch");
  BCUDA(cudaStreamSynchronize(b->stream), "batch synchronize");
  return MLBM_OK;
}

mlbm_status mlbm_batch_set_tuning(mlbm_batch* b, int32_t rows_density,
                                  int32_t rows_update, int32_t planes,
                                  int32_t blocks_per_sm, int32_t use_graphs) {
  if (!b) return bfail(MLBM_ERR_ARG, "null batch");
  auto ok_rows = [](int r) { return r == 1 || r == 2 || r == 4 || r == 8; };
  if (!ok_rows(rows_density) || !ok_rows(rows_update) || planes < 1 ||
      planes > 1024 || blocks_per_sm < 0 || blocks_per_sm > 32)
    return bfail(MLBM_ERR_ARG, "invalid batch tuning");
  BCUDA(cudaStreamSynchronize(b->stream), "batch tuning");
  b->By_d = rows_density;
  b->By_u = rows_update;
  b->Dz = planes;
  b->bps = blocks_per_sm;
  b->use_graphs = use_graphs ? 1 : 0;
  b->dirty = true;
  return MLBM_OK;
}

mlbm_status mlbm_batch_autotune(mlbm_batch* b, int32_t trial_steps,
                                int32_t* out) {
  if (!b) return bfail(MLBM_ERR_ARG, "null batch");
  if (trial_steps < 1) trial_steps = 2;
  if (b->dirty)
    if (mlbm_status st = rebuild(b)) return st;
  if (b->compact) {
    // one thread per node (pair) per pass: no work-item shape to tune
    if (out) {
      out[0] = b->By_d;
      out[1] = b->By_u;
      out[2] = b->Dz;
      out[3] = b->bps;
    }
    return MLBM_OK;
  }
  struct Cand { int bd, bu, dz, bps; };
  const Cand cands[] = {{4, 4, 8, 0},  {2, 2, 8, 0},  {8, 4, 8, 0},
                        {4, 4, 1, 0},  {4, 4, 32, 0}, {4, 2, 16, 0},
                        {8, 8, 8, 0},  {4, 4, 8, 4},  {2, 4, 4, 0}};
  float best = 1e30f;
  Cand pick = cands[0];
  cudaEvent_t e0, e1;
  BCUDA(cudaEventCreate(&e0), "autotune");
  BCUDA(cudaEventCreate(&e1), "autotune");
  for (const Cand& c : cands) {
    if (mlbm_status st = mlbm_batch_set_tuning(b, c.bd, c.bu, c.dz, c.bps, 0))
      return st;
    if (mlbm_status st = mlbm_batch_iterate(b, 1, 1, 0)) return st;  // warm-up
    cudaEventRecord(e0, b->stream);
    if (mlbm_status st = mlbm_batch_iterate(b, trial_steps, 1, 0)) return st;
    cudaEventRecord(e1, b->stream);
    BCUDA(cudaEventSynchronize(e1), "autotune");
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) {
      best = ms;
      pick = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (mlbm_status st = mlbm_batch_set_tuning(b, pick.bd, pick.bu, pick.dz, pick.bps, 1))
    return st;
  if (out) {
    out[0] = pick.bd;
    out[1] = pick.bu;
    out[2] = pick.dz;
    out[3] = pick.bps;
  }
  return MLBM_OK;
}

}  // extern "C"
