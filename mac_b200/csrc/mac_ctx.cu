// Context lifetime, host <-> device state transfer and the C-ABI entry points.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <utility>
#include <vector>

#include "mac_internal.cuh"

namespace mac {

int check(cudaError_t e) {
  if (e == cudaSuccess) return MAC_OK;
  if (e == cudaErrorMemoryAllocation) return MAC_ERR_OUT_OF_MEMORY;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return MAC_ERR_NO_DEVICE;
  return MAC_ERR_CUDA;
}

#define MAC_TRY(x)                 \
  do {                             \
    int rc_ = (x);                 \
    if (rc_ != MAC_OK) return rc_; \
  } while (0)
#define MAC_CUDA(x) MAC_TRY(check(x))

template <class T>
static int dalloc(T** p, size_t n) {
  return check(cudaMalloc((void**)p, sizeof(T) * (n ? n : 1)));
}

// ------------------------------------------------------------- kernels
__global__ void k_init_lists(int* blist, int* freelist, int nb, int cap) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nb) blist[i] = i;
  if (i >= nb && i < cap) freelist[i - nb] = cap - 1 - (i - nb);
}

__global__ void k_pack_lay(const uint8_t* __restrict__ ex, const int32_t* __restrict__ layer,
                           int8_t* __restrict__ lay, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) lay[i] = ex[i] ? (int8_t)layer[i] : kMissing;
}

// depth: int32 on the host, int16 in the pool (-1 empty; depths stay far below
// 2^15 in any world the pool holds)
__global__ void k_pack_depth(const int32_t* __restrict__ in, int16_t* __restrict__ out, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    int32_t v = in[i];
    out[i] = (int16_t)(v < -1 ? -1 : (v > 32766 ? 32766 : v));
  }
}

__global__ void k_unpack_depth(const int16_t* __restrict__ d, const int* __restrict__ blist, int nlive,
                               int32_t* __restrict__ out) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)nlive * kCells) return;
  out[i] = d[(size_t)blist[i >> 9] * kCells + (i & 511)];
}

__global__ void k_set_keys(int* bkey, const int32_t* __restrict__ keys, int nb) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 3 * nb) bkey[i] = keys[i];
}

__global__ void k_aos_to_soa(const double* __restrict__ aos, double* px, double* py, double* pz,
                             int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    px[i] = aos[3 * i];
    py[i] = aos[3 * i + 1];
    pz[i] = aos[3 * i + 2];
  }
}

__global__ void k_soa_to_aos(double* __restrict__ aos, const double* px, const double* py,
                             const double* pz, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    aos[3 * i] = px[i];
    aos[3 * i + 1] = py[i];
    aos[3 * i + 2] = pz[i];
  }
}

template <class T>
__global__ void k_gather_bricks(T* __restrict__ out, const T* __restrict__ in, const int* __restrict__ blist,
                                int nlive) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)nlive * kCells) return;
  int bi = (int)(i >> 9);
  int o = (int)(i & 511);
  out[i] = in[(size_t)blist[bi] * kCells + o];
}

// The inverse of k_gather_bricks: brick-ordered values into the pool.
__global__ void k_scatter_bricks(double* __restrict__ out, const double* __restrict__ in,
                                 const int* __restrict__ blist, int nlive) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)nlive * kCells) return;
  out[(size_t)blist[(int)(i >> 9)] * kCells + (i & 511)] = in[i];
}

__global__ void k_unpack_lay(const int8_t* __restrict__ lay, const int* __restrict__ blist, int nlive,
                             uint8_t* __restrict__ ex, int32_t* __restrict__ layer) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)nlive * kCells) return;
  int8_t l = lay[(size_t)blist[i >> 9] * kCells + (i & 511)];
  ex[i] = l != kMissing;
  layer[i] = l == kMissing ? -1 : l;
}

__global__ void k_gather_keys(int32_t* out, const int* bkey, const int* blist, int nlive) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 3 * nlive) out[i] = bkey[blist[i / 3] * 3 + i % 3];
}

// ------------------------------------------------------------- profiling
struct Prof {
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending[kPhases];
  std::vector<cudaEvent_t> spare;
  cudaEvent_t open[kPhases] = {};
  double ms[kPhases] = {};
  long long n[kPhases] = {};
};

static cudaEvent_t take_event(Prof* p) {
  if (!p->spare.empty()) {
    cudaEvent_t e = p->spare.back();
    p->spare.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

void prof_begin(Ctx* c, int ph) {
  if (!c->prof) return;
  cudaEvent_t e = take_event(c->prof);
  cudaEventRecord(e, c->stream);
  c->prof->open[ph] = e;
}

void prof_end(Ctx* c, int ph) {
  if (!c->prof || !c->prof->open[ph]) return;
  cudaEvent_t e = take_event(c->prof);
  cudaEventRecord(e, c->stream);
  c->prof->pending[ph].push_back({c->prof->open[ph], e});
  c->prof->open[ph] = nullptr;
}

static void prof_resolve(Ctx* c) {
  Prof* p = c->prof;
  if (!p) return;
  cudaStreamSynchronize(c->stream);
  for (int ph = 0; ph < kPhases; ++ph) {
    for (auto& pr : p->pending[ph]) {
      float ms = 0;
      cudaEventElapsedTime(&ms, pr.first, pr.second);
      p->ms[ph] += ms;
      p->n[ph] += 1;
      p->spare.push_back(pr.first);
      p->spare.push_back(pr.second);
    }
    p->pending[ph].clear();
  }
}

static void prof_free(Ctx* c) {
  Prof* p = c->prof;
  if (!p) return;
  prof_resolve(c);
  for (cudaEvent_t e : p->spare) cudaEventDestroy(e);
  delete p;
  c->prof = nullptr;
}

// ------------------------------------------------------------- lifetime
static void free_all(Ctx* c) {
  prof_free(c);
  free_solver(c);
  cudaFree(c->bkey); cudaFree(c->lay); cudaFree(c->type); cudaFree(c->flags); cudaFree(c->f64);
  cudaFree(c->pdir);
  cudaFree(c->depth); cudaFree(c->pkeep); cudaFree(c->u2);
  for (int k = 0; k < 2; ++k)
    for (int i = 0; i < 3; ++i) { cudaFree(c->pbuf[k][i]); cudaFree(c->pbuf2[k][i]); }
  cudaFree(c->nbr); cudaFree(c->blist); cudaFree(c->blist2); cudaFree(c->freelist); cudaFree(c->alive);
  cudaFree(c->hkeys); cudaFree(c->hval); cudaFree(c->newslots);
  cudaFree(c->px); cudaFree(c->py); cudaFree(c->pz); cudaFree(c->pending);
  cudaFree(c->px2); cudaFree(c->py2); cudaFree(c->pz2); cudaFree(c->pbrick);
  cudaFree(c->bcount); cudaFree(c->bcursor); cudaFree(c->boff); cudaFree(c->lmask);
  cudaFree(c->ds);
  if (c->hs) cudaFreeHost(c->hs);
  if (c->hs_lag) cudaFreeHost(c->hs_lag);
  for (cudaEvent_t e : c->ev_lag)
    if (e) cudaEventDestroy(e);
  if (c->ev_topo) cudaEventDestroy(c->ev_topo);
  if (c->ev_bins) cudaEventDestroy(c->ev_bins);
  if (c->side) cudaStreamDestroy(c->side);
  cudaFree(c->csc_off); cudaFree(c->csc_ind); cudaFree(c->csc_val); cudaFree(c->csc_vec);
  cudaFree(c->csr_off); cudaFree(c->csr_ind); cudaFree(c->csr_val); cudaFree(c->eb_work);
  if (c->stream) cudaStreamDestroy(c->stream);
}

static int create(const mac_params* p, Ctx** out) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MAC_ERR_NO_DEVICE;
  if (!p || p->max_bricks <= 0 || p->max_particles < 0 || p->layer_max < 0 || p->layer_max > 120 ||
      p->gravity_axis < 1 || p->gravity_axis > 3)
    return MAC_ERR_INVALID;
  for (int i = 0; i < 3; ++i)
    if (!(p->h[i] > 0)) return MAC_ERR_INVALID;
  if (!(p->viscosity >= 0) || !std::isfinite(p->viscosity)) return MAC_ERR_INVALID;
  if (p->refill_cube < 0 || p->refill_cube > 4) return MAC_ERR_INVALID;
  if (p->depth_mode && (p->depth_interior < 0 || p->depth_remove < 0)) return MAC_ERR_INVALID;
  if (p->pipeline < 0 || p->pipeline > 1 || (p->pipeline == 1 && !p->depth_mode)) return MAC_ERR_INVALID;
  if (p->device < 0 || p->device >= ndev) return MAC_ERR_INVALID;
  MAC_CUDA(cudaSetDevice(p->device));
  Ctx* c = new (std::nothrow) Ctx();
  if (!c) return MAC_ERR_OUT_OF_MEMORY;
  c->prm = *p;
  for (int i = 0; i < 3; ++i) {
    c->dp.h[i] = p->h[i];
    c->dp.ih[i] = 1 / p->h[i];  // Inversible_Value::Inverse (src/Inversible_Value_Vect.h:9-16)
    c->dp.ih2[i] = c->dp.ih[i] * c->dp.ih[i];
  }
  for (int az = 0; az < 3; ++az)
    for (int ay = 0; ay < 3; ++ay)
      for (int ax = 0; ax < 3; ++ax) {
        double d = ax * c->dp.ih2[0] + ay * c->dp.ih2[1] + az * c->dp.ih2[2];
        c->dp.dtab[ax + 3 * ay + 9 * az] = d > 0 ? 1.0 / d : 0.0;
      }
  // multigrid smoother (mac_set_smoother): the two sweep weights are the
  // reciprocals of the degree-2 Chebyshev roots on [0.3, 2] (the spectrum of
  // D^-1 A lies in (0, 2]); they took the 256^3 pool at 1e-8 from 17 to 15
  // CG iterations against two sweeps at 0.9
  c->dp.mgw1 = 0.5711;
  c->dp.mgw2 = 1.8216;
  c->dp.mgws = 0.9;
  c->dp.cfl = p->cfl_factor;
  c->dp.dt_min = p->dt_min;
  c->dp.dt_max = p->dt_max;
  c->dp.g = p->gravity;
  c->dp.gaxis = p->gravity_axis - 1;
  c->dp.layer_max = p->layer_max;
  c->dp.interp_sym = p->interp_symmetric;
  c->dp.nu = p->viscosity;
  c->dp.depth_mode = p->depth_mode ? 1 : 0;
  c->dp.depth_interior = p->depth_interior;
  c->dp.depth_remove = p->depth_remove;
  c->dp.refill_cube = p->refill_cube;
  c->dp.pipeline = p->pipeline;
  for (int i = 0; i < 3; ++i) c->dp.lih2[i] = std::pow(c->dp.ih[i], 2);
  c->cap_bricks = p->max_bricks;
  c->cap_particles = p->max_particles;
  c->hcap = 64;
  while (c->hcap < 4 * c->cap_bricks) c->hcap <<= 1;
  c->cap_pending = c->cap_particles < (1 << 22) ? (c->cap_particles + 1) : (1 << 22);
  size_t nc = (size_t)c->cap_bricks * kCells;
  int rc = MAC_OK;
  auto A = [&](int r) { if (rc == MAC_OK) rc = r; };
  // the context's stream at the highest priority, the side stream (particle
  // binning beside the solve) at the lowest: the block scheduler serves the
  // solve's kernels first and the binning fills what they leave
  int prio_low = 0, prio_high = 0;
  A(check(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high)));
  A(check(cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, prio_high)));
  A(check(cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, prio_low)));
  A(check(cudaEventCreateWithFlags(&c->ev_topo, cudaEventDisableTiming)));
  A(check(cudaEventCreateWithFlags(&c->ev_bins, cudaEventDisableTiming)));
  A(dalloc(&c->bkey, 3 * c->cap_bricks));
  A(dalloc(&c->lay, nc));
  A(dalloc(&c->type, nc));
  A(dalloc(&c->flags, nc));
  A(dalloc(&c->f64, NF64 * nc));
  if (p->viscosity > 0) A(dalloc(&c->pdir, nc));
  if (p->depth_mode) {
    A(dalloc(&c->depth, nc));
    A(dalloc(&c->pkeep, (size_t)c->cap_particles));
  }
  if (p->pipeline == 1) {
    A(dalloc(&c->u2, 3 * nc));
    for (int k = 0; k < 2; ++k)
      for (int i = 0; i < 3; ++i) {
        A(dalloc(&c->pbuf[k][i], (size_t)c->cap_particles));
        A(dalloc(&c->pbuf2[k][i], (size_t)c->cap_particles));
      }
  }
  A(dalloc(&c->nbr, kNbr * c->cap_bricks));
  A(dalloc(&c->blist, c->cap_bricks));
  A(dalloc(&c->blist2, c->cap_bricks));
  A(dalloc(&c->freelist, c->cap_bricks));
  A(dalloc(&c->alive, c->cap_bricks));
  A(dalloc(&c->hkeys, c->hcap));
  A(dalloc(&c->hval, c->hcap));
  A(dalloc(&c->newslots, c->cap_bricks + 1));
  A(dalloc(&c->px, c->cap_particles));
  A(dalloc(&c->py, c->cap_particles));
  A(dalloc(&c->pz, c->cap_particles));
  A(dalloc(&c->pending, c->cap_pending));
  A(dalloc(&c->px2, c->cap_particles));
  A(dalloc(&c->py2, c->cap_particles));
  A(dalloc(&c->pz2, c->cap_particles));
  A(dalloc(&c->pbrick, c->cap_particles));
  A(dalloc(&c->bcount, c->cap_bricks + 1));
  A(dalloc(&c->lmask, c->cap_bricks));
  A(dalloc(&c->bcursor, (size_t)(c->cap_bricks + 1) * kCells));
  A(dalloc(&c->boff, c->cap_bricks + 2));
  A(dalloc(&c->ds, 1));
  if (rc == MAC_OK) A(check(cudaMallocHost((void**)&c->hs, sizeof(Scalars))));
  if (rc == MAC_OK) A(check(cudaMallocHost((void**)&c->hs_lag, 2 * sizeof(Scalars))));
  for (int k = 0; k < 2 && rc == MAC_OK; ++k) A(check(cudaEventCreateWithFlags(&c->ev_lag[k], cudaEventDisableTiming)));
  if (rc == MAC_OK) A(alloc_solver(c));
  if (rc == MAC_OK) {
    A(check(cudaMemsetAsync(c->ds, 0, sizeof(Scalars), c->stream)));
    A(check(cudaMemsetAsync(c->lay, 0xFE, nc, c->stream)));  // -2: missing
  }
  if (rc != MAC_OK) {
    free_all(c);
    delete c;
    return rc;
  }
  *out = c;
  return MAC_OK;
}

int read_scalars(Ctx* c) {
  MAC_CUDA(cudaMemcpyAsync(c->hs, c->ds, sizeof(Scalars), cudaMemcpyDeviceToHost, c->stream));
  MAC_CUDA(cudaStreamSynchronize(c->stream));
  c->nlive_host = c->hs->nlive;
  c->np_host = c->hs->np;
  c->stats.live_bricks = c->hs->nlive;
  c->stats.particles = c->hs->np;
  if (c->hs->err) {
    if (c->hs->err & (kErrBricks | kErrParticles | kErrHash | kErrPending)) return MAC_ERR_CAPACITY;
    if (c->hs->err & kErrTimeout) return MAC_ERR_TIMEOUT;
    return MAC_ERR_INVALID;
  }
  return MAC_OK;
}

static int upload(Ctx* c, const mac_host_state* s) {
  if (!s || s->nbricks < 0 || s->nparticles < 0) return MAC_ERR_INVALID;
  if (s->nbricks > c->cap_bricks || s->nparticles > c->cap_particles) return MAC_ERR_CAPACITY;
  int nb = (int)s->nbricks;
  size_t nc = (size_t)nb * kCells, cap = (size_t)c->cap_bricks * kCells;
  cudaStream_t st = c->stream;
  if (nb > 0) {
    // keys through a staging area (solver vector r), then the fields straight into the pool.
    int32_t* tkeys = (int32_t*)c->r;
    MAC_CUDA(cudaMemcpyAsync(tkeys, s->keys, sizeof(int32_t) * 3 * nb, cudaMemcpyHostToDevice, st));
    k_set_keys<<<grid_for(3 * nb, 256), 256, 0, st>>>(c->bkey, tkeys, nb); MAC_COUNT(c);
    // a NULL stage buffer (speed 1, acceleration) is not transferred: zeroed here
    for (int f = 0; f < NF64; ++f) {
      const double* src = f < 6 ? s->u[f / 3][f % 3] : (f < 9 ? s->acc[f - 6] : s->p);
      double* dst = c->f64 + (size_t)f * cap;
      if (src) MAC_CUDA(cudaMemcpyAsync(dst, src, 8 * nc, cudaMemcpyHostToDevice, st));
      else MAC_CUDA(cudaMemsetAsync(dst, 0, 8 * nc, st));
    }
    MAC_CUDA(cudaMemcpyAsync(c->flags, s->flags, nc, cudaMemcpyHostToDevice, st));
    MAC_CUDA(cudaMemcpyAsync(c->type, s->type, nc, cudaMemcpyHostToDevice, st));
    uint8_t* tex = (uint8_t*)c->z;
    int32_t* tlay = (int32_t*)c->q;
    MAC_CUDA(cudaMemcpyAsync(tex, s->exists, nc, cudaMemcpyHostToDevice, st));
    MAC_CUDA(cudaMemcpyAsync(tlay, s->layer, 4 * nc, cudaMemcpyHostToDevice, st));
    k_pack_lay<<<grid_for((int64_t)nc, 256), 256, 0, st>>>(tex, tlay, c->lay, (int64_t)nc); MAC_COUNT(c);
    if (c->depth && s->depth) {
      MAC_CUDA(cudaMemcpyAsync(tlay, s->depth, 4 * nc, cudaMemcpyHostToDevice, st));
      k_pack_depth<<<grid_for((int64_t)nc, 256), 256, 0, st>>>(tlay, c->depth, (int64_t)nc); MAC_COUNT(c);
    } else if (c->depth) {
      MAC_CUDA(cudaMemsetAsync(c->depth, 0xFF, 2 * nc, st));
    }
  }
  if (cap > nc) MAC_CUDA(cudaMemsetAsync(c->lay + nc, 0xFE, cap - nc, st));
  if (cap > nc && c->depth) MAC_CUDA(cudaMemsetAsync(c->depth + nc, 0xFF, 2 * (cap - nc), st));
  // speed buffer 2 is not part of a state: the prototype value everywhere
  if (c->u2) MAC_CUDA(cudaMemsetAsync(c->u2, 0, 8 * 3 * cap, st));
  c->imove = 0;
  k_init_lists<<<grid_for(c->cap_bricks, 256), 256, 0, st>>>(c->blist, c->freelist, nb, (int)c->cap_bricks); MAC_COUNT(c);
  // particles, through a bounded staging buffer (solver vector pd)
  int64_t np = s->nparticles;
  int64_t chunk = (int64_t)(cap / 3);
  for (int64_t o = 0; o < np; o += chunk) {
    int64_t n = np - o < chunk ? np - o : chunk;
    MAC_CUDA(cudaMemcpyAsync(c->pd, s->pos + 3 * o, 24 * n, cudaMemcpyHostToDevice, st));
    k_aos_to_soa<<<grid_for(n, 256), 256, 0, st>>>(c->pd, c->px + o, c->py + o, c->pz + o, n); MAC_COUNT(c);
  }
  Scalars h{};
  h.nlive = nb;
  h.nfree = (int)(c->cap_bricks - nb);
  h.np = np;
  h.dt = s->dt;
  h.t = s->t;
  std::memcpy(c->hs, &h, sizeof(h));
  MAC_CUDA(cudaMemcpyAsync(c->ds, c->hs, sizeof(Scalars), cudaMemcpyHostToDevice, st));
  c->seed = s->step;
  c->nlive_host = nb;
  c->np_host = np;
  c->system_ready = false;
  MAC_TRY(rebuild_index(c));
  return read_scalars(c);
}

static int download(Ctx* c, mac_host_state* s) {
  MAC_TRY(read_scalars(c));
  int nb = c->nlive_host;
  if (!s || s->nbricks < nb || s->nparticles < c->np_host) return MAC_ERR_INVALID;
  size_t nc = (size_t)nb * kCells, cap = (size_t)c->cap_bricks * kCells;
  cudaStream_t st = c->stream;
  double* tmp = c->r;  // staging
  int g = grid_for((int64_t)nc, 256);
  if (nb > 0) {
    int32_t* tk = (int32_t*)c->z;
    k_gather_keys<<<grid_for(3 * nb, 256), 256, 0, st>>>(tk, c->bkey, c->blist, nb); MAC_COUNT(c);
    MAC_CUDA(cudaMemcpyAsync(s->keys, tk, 12 * (size_t)nb, cudaMemcpyDeviceToHost, st));
    for (int f = 0; f < NF64; ++f) {
      double* dst = f < 6 ? s->u[f / 3][f % 3] : (f < 9 ? s->acc[f - 6] : s->p);
      if (!dst) continue;  // a field the caller leaves out
      k_gather_bricks<double><<<g, 256, 0, st>>>(tmp, c->f64 + (size_t)f * cap, c->blist, nb); MAC_COUNT(c);
      MAC_CUDA(cudaMemcpyAsync(dst, tmp, 8 * nc, cudaMemcpyDeviceToHost, st));
      MAC_CUDA(cudaStreamSynchronize(st));
    }
    uint8_t* t8 = (uint8_t*)c->z;
    k_gather_bricks<uint8_t><<<g, 256, 0, st>>>(t8, c->flags, c->blist, nb); MAC_COUNT(c);
    MAC_CUDA(cudaMemcpyAsync(s->flags, t8, nc, cudaMemcpyDeviceToHost, st));
    MAC_CUDA(cudaStreamSynchronize(st));
    k_gather_bricks<uint8_t><<<g, 256, 0, st>>>(t8, c->type, c->blist, nb); MAC_COUNT(c);
    MAC_CUDA(cudaMemcpyAsync(s->type, t8, nc, cudaMemcpyDeviceToHost, st));
    MAC_CUDA(cudaStreamSynchronize(st));
    int32_t* tl = (int32_t*)c->q;
    k_unpack_lay<<<g, 256, 0, st>>>(c->lay, c->blist, nb, t8, tl); MAC_COUNT(c);
    MAC_CUDA(cudaMemcpyAsync(s->exists, t8, nc, cudaMemcpyDeviceToHost, st));
    MAC_CUDA(cudaMemcpyAsync(s->layer, tl, 4 * nc, cudaMemcpyDeviceToHost, st));
    if (s->depth && c->depth) {
      k_unpack_depth<<<g, 256, 0, st>>>(c->depth, c->blist, nb, tl); MAC_COUNT(c);
      MAC_CUDA(cudaMemcpyAsync(s->depth, tl, 4 * nc, cudaMemcpyDeviceToHost, st));
    } else if (s->depth) {
      for (size_t i = 0; i < nc; ++i) s->depth[i] = -1;
    }
  }
  int64_t np = c->np_host;
  int64_t chunk = (int64_t)(cap / 3);
  for (int64_t o = 0; o < np; o += chunk) {
    int64_t n = np - o < chunk ? np - o : chunk;
    k_soa_to_aos<<<grid_for(n, 256), 256, 0, st>>>(c->pd, c->px + o, c->py + o, c->pz + o, n); MAC_COUNT(c);
    MAC_CUDA(cudaMemcpyAsync(s->pos + 3 * o, c->pd, 24 * n, cudaMemcpyDeviceToHost, st));
    MAC_CUDA(cudaStreamSynchronize(st));
  }
  MAC_CUDA(cudaStreamSynchronize(st));
  s->nbricks = nb;
  s->nparticles = np;
  s->t = c->hs->t;
  s->dt = c->hs->dt;
  s->step = c->seed;
  return MAC_OK;
}

// One FP64 cell field (MAC_FIELD_*) of every live brick, in the brick order of
// mac_download_state (the order of the last upload while no topology pass has
// run), through the solver vector q as staging.
int field_transfer(Ctx* c, int field, const double* hin, double* hout) {
  if (field < 0 || field >= NF64) return MAC_ERR_INVALID;
  MAC_TRY(read_scalars(c));
  const int nb = c->nlive_host;
  if (nb == 0) return MAC_OK;
  const size_t nc = (size_t)nb * kCells, cap = (size_t)c->cap_bricks * kCells;
  cudaStream_t st = c->stream;
  double* dst = c->f64 + (size_t)field * cap;
  const int g = grid_for((int64_t)nc, 256);
  if (hin) {
    MAC_CUDA(cudaMemcpyAsync(c->q, hin, 8 * nc, cudaMemcpyHostToDevice, st));
    k_scatter_bricks<<<g, 256, 0, st>>>(dst, c->q, c->blist, nb); MAC_COUNT(c);
  } else {
    k_gather_bricks<double><<<g, 256, 0, st>>>(c->q, dst, c->blist, nb); MAC_COUNT(c);
    MAC_CUDA(cudaMemcpyAsync(hout, c->q, 8 * nc, cudaMemcpyDeviceToHost, st));
  }
  MAC_CUDA(cudaStreamSynchronize(st));
  return MAC_OK;
}

}  // namespace mac

using mac::Ctx;

extern "C" {

void mac_default_params(mac_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->h[0] = p->h[1] = p->h[2] = 0.05;
  p->cfl_factor = 0.5;
  p->dt_min = 0.0;
  p->dt_max = 0.1;
  p->gravity = -9.81;
  p->gravity_axis = 3;
  p->layer_max = 4;
  p->interp_symmetric = 1;
  p->solver = MAC_SOLVER_MGPCG_FP64;
  p->rtol = 1e-8;
  p->max_iters = 500;
  p->warm_start = 0;
  p->max_bricks = 4096;
  p->max_particles = 1 << 20;
  p->device = 0;
  p->div_check = 1;
}

const char* mac_error_string(int code) {
  switch (code) {
    case MAC_OK: return "ok";
    case MAC_ERR_INVALID: return "invalid argument or state";
    case MAC_ERR_CUDA: return "CUDA error";
    case MAC_ERR_CAPACITY: return "capacity exceeded (bricks, particles or hash table)";
    case MAC_ERR_NOT_CONVERGED: return "solver did not converge";
    case MAC_ERR_NO_DEVICE: return "no CUDA device";
    case MAC_ERR_OUT_OF_MEMORY: return "out of device memory";
    case MAC_ERR_TIMEOUT: return "timeout";
    case MAC_ERR_MATRIX: return "matrix not of the form the solver handles";
    default: return "unknown error";
  }
}

int mac_ctx_create(const mac_params* p, void** ctx) {
  if (!ctx) return MAC_ERR_INVALID;
  Ctx* c = nullptr;
  int rc = mac::create(p, &c);
  *ctx = c;
  return rc;
}

int mac_ctx_destroy(void* ctx) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MAC_ERR_INVALID;
  cudaSetDevice(c->prm.device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  mac::free_all(c);
  delete c;
  return MAC_OK;
}

int mac_get_stats(void* ctx, mac_stats* out) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !out) return MAC_ERR_INVALID;
  *out = c->stats;
  return MAC_OK;
}

int mac_upload_state(void* ctx, const mac_host_state* s) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MAC_ERR_INVALID;
  cudaSetDevice(c->prm.device);
  return mac::upload(c, s);
}

int mac_query_sizes(void* ctx, int64_t* nbricks, int64_t* nparticles) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MAC_ERR_INVALID;
  int rc = mac::read_scalars(c);
  if (nbricks) *nbricks = c->nlive_host;
  if (nparticles) *nparticles = c->np_host;
  return rc;
}

int mac_upload_field(void* ctx, int field, const double* data) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !data) return MAC_ERR_INVALID;
  cudaSetDevice(c->prm.device);
  return mac::field_transfer(c, field, data, nullptr);
}

int mac_download_field(void* ctx, int field, double* data) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !data) return MAC_ERR_INVALID;
  cudaSetDevice(c->prm.device);
  return mac::field_transfer(c, field, nullptr, data);
}

int mac_download_state(void* ctx, mac_host_state* s) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MAC_ERR_INVALID;
  cudaSetDevice(c->prm.device);
  return mac::download(c, s);
}

int mac_sync(void* ctx) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MAC_ERR_INVALID;
  return mac::check(cudaStreamSynchronize(c->stream));
}

int mac_stream(void* ctx, void** stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !stream) return MAC_ERR_INVALID;
  *stream = (void*)c->stream;
  return MAC_OK;
}

int mac_launch_count(void* ctx, int64_t* count) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !count) return MAC_ERR_INVALID;
  *count = c->launches;
  return MAC_OK;
}

int mac_set_profiling(void* ctx, int on) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MAC_ERR_INVALID;
  if (on && !c->prof) c->prof = new (std::nothrow) mac::Prof();
  if (!on) mac::prof_free(c);
  return (on && !c->prof) ? MAC_ERR_OUT_OF_MEMORY : MAC_OK;
}

int mac_get_profile(void* ctx, double* ms, int64_t* count, int nphase) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !ms || !count || nphase <= 0) return MAC_ERR_INVALID;
  mac::prof_resolve(c);
  for (int i = 0; i < nphase; ++i) {
    bool have = c->prof && i < mac::kPhases;
    ms[i] = have ? c->prof->ms[i] : 0.0;
    count[i] = have ? c->prof->n[i] : 0;
  }
  if (c->prof)
    for (int i = 0; i < mac::kPhases; ++i) {
      c->prof->ms[i] = 0;
      c->prof->n[i] = 0;
    }
  return MAC_OK;
}

}  // extern "C"
