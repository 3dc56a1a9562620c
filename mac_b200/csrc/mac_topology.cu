// Topology rebuild on the device: the integer passes of the per-step init
// sequence Algorithms<Initialize_MacCell, Layer_Initial_With_Particle,
// Create_Fluid_Particle, Update_CellType_Layer, Delete_MacCell,
// Calculate_Time_Step> (test/TestJetDEau_Basic.cpp:325-326), bit-exact with
// the reference, plus the index maintenance of the brick pool. With
// depth_mode the same kernels run the depth composition of test/Jet3.cpp:519-549
// (Initialize_Layer_And_Depth, Layer_Initial_With_Particle_Depth,
// Create_Fluid_Particle_Depth, Update_CellType_Layer_Depth): cells carry a
// depth and deep fluid becomes the interior material.
//
// Cell creation (the reference's auto-creating operator[],
// src/ChunkHashTable.tpp:62-87) is split in two so that no thread ever waits
// on another: a pass inserts the missing brick keys into the hash table, a
// second kernel gives each new key a pool brick initialised to the prototype
// (speed 0, pressure 0, air, no flags, no existing cell), and the pass that
// needed the cells runs again.
#include <utility>

#include "mac_internal.cuh"

namespace mac {

constexpr int kTopoBlocks = 1184;  // 8 x 148 SMs, grid-stride over bricks

// --------------------------------------------------------------- hashing
__device__ int hash_insert(unsigned long long* hk, int64_t hcap, unsigned long long key, int* newslots,
                           Scalars* ds, int64_t cap_new) {
  unsigned long long s = hmix(key) & (unsigned long long)(hcap - 1);
  for (int64_t probe = 0; probe < hcap; ++probe) {
    unsigned long long k = hk[s];
    if (k == key) return (int)s;
    if (k == kEmptyKey) {
      unsigned long long old = atomicCAS(hk + s, kEmptyKey, key);
      if (old == kEmptyKey) {
        int pos = atomicAdd(&ds->nnew, 1);
        if (pos < cap_new) newslots[pos] = (int)s;
        else atomicOr(&ds->err, kErrBricks);
        return (int)s;
      }
      if (old == key) return (int)s;
    }
    s = (s + 1) & (unsigned long long)(hcap - 1);
  }
  atomicOr(&ds->err, kErrHash);
  return -1;
}

__global__ void k_hash_clear(unsigned long long* hk, int* hv, int64_t hcap) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < hcap) {
    hk[i] = kEmptyKey;
    hv[i] = kPending;
  }
}

__global__ void k_hash_insert_live(const int* __restrict__ blist, const int* __restrict__ bkey,
                                   unsigned long long* hk, int* hv, int64_t hcap, Scalars* ds) {
  int n = ds->nlive;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int b = blist[i];
    unsigned long long key = pack_key(bkey[3 * b], bkey[3 * b + 1], bkey[3 * b + 2]);
    unsigned long long s = hmix(key) & (unsigned long long)(hcap - 1);
    bool ok = false;
    for (int64_t probe = 0; probe < hcap; ++probe) {
      if (atomicCAS(hk + s, kEmptyKey, key) == kEmptyKey) {
        hv[s] = b;
        ok = true;
        break;
      }
      s = (s + 1) & (unsigned long long)(hcap - 1);
    }
    if (!ok) atomicOr(&ds->err, kErrHash);
  }
}

__global__ void k_build_nbr(const int* __restrict__ blist, const int* __restrict__ bkey,
                            const unsigned long long* __restrict__ hk, const int* __restrict__ hv,
                            int64_t hcap, int* __restrict__ nbr, Scalars* ds) {
  int n = ds->nlive;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (int64_t)n * kNbr;
       i += (int64_t)gridDim.x * blockDim.x) {
    int b = blist[i / kNbr];
    int d = (int)(i % kNbr);
    int dx = d % 3 - 1, dy = (d / 3) % 3 - 1, dz = d / 9 - 1;
    int r = (d == kSelf) ? b
                         : hash_find(hk, hv, hcap, pack_key(bkey[3 * b] + dx, bkey[3 * b + 1] + dy, bkey[3 * b + 2] + dz));
    nbr[(size_t)b * kNbr + d] = r < 0 ? -1 : r;
  }
}

__global__ void k_bbox(const int* __restrict__ blist, const int* __restrict__ bkey, Scalars* ds) {
  int n = ds->nlive;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int b = blist[i];
    for (int a = 0; a < 3; ++a) {
      atomicMin(&ds->bbox[a], bkey[3 * b + a]);
      atomicMax(&ds->bbox[3 + a], bkey[3 * b + a]);
    }
  }
}

__global__ void k_bbox_reset(Scalars* ds) {
  for (int a = 0; a < 3; ++a) {
    ds->bbox[a] = 0x3fffffff;
    ds->bbox[3 + a] = -0x3fffffff;
  }
}

// New hash slots get a pool brick initialised to the prototype chunk
// (Data_Chunk::Allocate copies the prototype cell into every slot:
// src/Data_Chunk_Base.h:20-29, src/Data_Chunk_Speed.h:99-123).
__global__ void k_alloc_bricks(const int* __restrict__ newslots, const unsigned long long* __restrict__ hk,
                               int* hv, int* bkey, int* blist, const int* __restrict__ freelist,
                               int8_t* lay, uint8_t* type, uint8_t* flags, double* f64, int16_t* depth,
                               double* u2, size_t cap_cells, int64_t cap_bricks, Scalars* ds) {
  __shared__ int sb;
  int n = ds->nnew;
  if (n > cap_bricks) n = (int)cap_bricks;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    if (threadIdx.x == 0) {
      int slot_i = newslots[i];
      int fi = atomicSub(&ds->nfree, 1) - 1;
      int b = -1;
      if (fi >= 0) {
        b = freelist[fi];
        int x, y, z;
        unpack_key(hk[slot_i], &x, &y, &z);
        bkey[3 * b] = x;
        bkey[3 * b + 1] = y;
        bkey[3 * b + 2] = z;
        int pos = atomicAdd(&ds->nlive, 1);
        blist[pos] = b;
      } else {
        atomicOr(&ds->err, kErrBricks);
      }
      hv[slot_i] = b;
      sb = b;
    }
    __syncthreads();
    int b = sb;
    if (b >= 0) {
      for (int o = threadIdx.x; o < kCells; o += blockDim.x) {
        size_t c = (size_t)b * kCells + o;
        lay[c] = kMissing;
        type[c] = MAC_CELL_AIR;
        flags[c] = 0;
        if (depth) depth[c] = -1;
        if (u2)
          for (int f = 0; f < 3; ++f) u2[(size_t)f * cap_cells + c] = 0.0;
        for (int f = 0; f < NF64; ++f) f64[(size_t)f * cap_cells + c] = 0.0;
      }
    }
    __syncthreads();
  }
}

__global__ void k_after_alloc(Scalars* ds) {
  if (ds->nfree < 0) ds->nfree = 0;
  ds->nnew = 0;
}

// ------------------------------------------------- Initialize_MacCell
// src/Algorithms_Initialize_MacCell.h:15-21: every existing cell -> empty layer.
// Depth composition (src/Algorithms_Initialize_Layer_And_Depth.h:16-33): also
// fluid cells that are not interior lose their depth.
__global__ void k_initialize(const int* __restrict__ blist, int8_t* lay, const uint8_t* __restrict__ type,
                             int16_t* depth, Scalars* ds) {
  int n = ds->nlive;
  for (int bi = blockIdx.x; bi < n; bi += gridDim.x) {
    size_t base = (size_t)blist[bi] * kCells;
    for (int o = threadIdx.x; o < kCells; o += blockDim.x) {
      if (lay[base + o] == kMissing) continue;
      lay[base + o] = kEmpty;
      if (depth) {
        uint8_t t = type[base + o];
        if (is_fluid(t) && t != MAC_CELL_INTERIOR) depth[base + o] = -1;
      }
    }
  }
}

// ------------------------------------- Layer_Initial_With_Particle
// src/Algorithms_Layer_Initial_With_Particle.h:26-30 with
// Policy_Particle_To_Key::GetKeyFromParticle (src/Policy_Particle_To_Key.h:24-35):
// key_i = lround(pos_i * (1/h_i)); grid[key] -> layer 0, SetFluid (air -> fluid only,
// src/Data_CellType_Fluid_Air_Solid_Inflow.tpp:150-157). Depth composition
// (src/Algorithms_Layer_Initial_With_Particle_Depth.h:26-47): a particle in an
// interior cell gives it layer 0 and keeps the material; it is marked for
// removal (pkeep = 0) when the cell is deeper than the removal depth. The
// marks depend only on state no thread of this pass changes (air -> fluid
// never makes an interior cell), so the passes are order-free.
__global__ void k_mark_particles(const double* __restrict__ px, const double* __restrict__ py,
                                 const double* __restrict__ pz, Params P, unsigned long long* hk, int* hv,
                                 int64_t hcap, int* newslots, int64_t cap_new, int8_t* lay, uint8_t* type,
                                 const int16_t* __restrict__ depth, uint8_t* pkeep, Scalars* ds, int pass) {
  if (pass == 1 && ds->done == 0) return;  // no brick was missing in pass 0
  int64_t n = ds->np;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    int kx = (int)lround(px[q] * P.ih[0]);
    int ky = (int)lround(py[q] * P.ih[1]);
    int kz = (int)lround(pz[q] * P.ih[2]);
    unsigned long long key = pack_key(fdiv8(kx), fdiv8(ky), fdiv8(kz));
    int b = hash_find(hk, hv, hcap, key);
    if (b < 0) {
      if (pass == 0) hash_insert(hk, hcap, key, newslots, ds, cap_new);
      else atomicOr(&ds->err, kErrBricks);
      if (pkeep) pkeep[q] = 1;  // a new cell is air, never interior
      continue;
    }
    size_t c = (size_t)b * kCells + (kx & 7) + 8 * (ky & 7) + 64 * (kz & 7);
    lay[c] = 0;
    uint8_t t = type[c];
    if (pkeep && t == MAC_CELL_INTERIOR) {
      pkeep[q] = depth[c] > P.depth_remove ? 0 : 1;
    } else {
      if (t == MAC_CELL_AIR) type[c] = MAC_CELL_FLUID;
      if (pkeep) pkeep[q] = 1;
    }
  }
}

// Removal of the marked particles (the list erase of
// src/Algorithms_Layer_Initial_With_Particle_Depth.h:33-36): kept particles are
// packed into the second position arrays with one atomic per warp. The order
// changes; nothing depends on the particle order.
// Up to three position buffers (pipeline B carries positions 0..2 of every
// particle) move together.
struct PartMove {
  const double* src[9];
  double* dst[9];
  int n;  // 3 or 9 arrays
};

__global__ void k_compact_particles(PartMove M, const uint8_t* __restrict__ pkeep, Scalars* ds) {
  const int64_t n = ds->np;
  const int lane = threadIdx.x & 31;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = base + threadIdx.x;
    const bool keep = q < n && pkeep[q];
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    unsigned long long w = 0;
    if (lane == 0 && m) w = atomicAdd(&ds->np_new, (unsigned long long)__popc(m));
    w = __shfl_sync(0xffffffffu, w, 0);
    if (keep) {
      const unsigned long long i = w + __popc(m & ((1u << lane) - 1u));
      for (int a = 0; a < M.n; ++a) M.dst[a][i] = M.src[a][q];
    }
  }
}

__global__ void k_compact_particles_done(Scalars* ds) {
  ds->np = (int64_t)ds->np_new;
  ds->np_new = 0;
}

// Remembers across the alloc kernel whether pass 1 of the particle marking must run.
__global__ void k_note_missing(Scalars* ds) { ds->done = ds->nnew > 0 ? 1 : 0; }
__global__ void k_clear_note(Scalars* ds) { ds->done = 0; }

// ------------------------------------------------ Create_Fluid_Particle
// Same jitter as the oracle's restatement: splitmix64 over (seed, key, slot, axis).
__device__ inline unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ inline void jitter8(unsigned long long seed, int kx, int ky, int kz, int s, const Params& P,
                               double out[3]) {
  int k[3] = {kx, ky, kz};
  unsigned long long base =
      mix64(seed ^ mix64(((unsigned long long)(uint32_t)kx) | ((unsigned long long)(uint32_t)ky << 32)));
  base = mix64(base ^ (unsigned long long)(uint32_t)kz);
  for (int i = 0; i < 3; ++i) {
    unsigned long long r = mix64(base ^ (unsigned long long)(s * 3 + i + 1));
    double u = (double)(r >> 11) * (1.0 / 9007199254740992.0);
    double j = (u - 0.5) * 0.499;
    double o = ((s >> i) & 1) ? 0.25 : -0.25;
    out[i] = (((double)k[i] + o) + j) * P.h[i];
  }
}

// src/Algorithms_Create_Fluid_Particle.h:25-33 with
// Policy_Is_Inbound_Filling_Layer_CellType (src/Policy_Is_Inbound_Filling_Layer_CellType.h:16-19):
// inflow cells whose layer is still empty are refilled and get layer 0 (SetFluid
// leaves an inflow cell inflow). The refill is 8 jittered particles, or
// Policy_Add_Particle_Cube(n) (src/Policy_Add_Particle_Cube.h:29-59): (2n+1)^3
// particles at (k_i + t_i/(2n+1)) h_i, t_i = -n..n. Depth composition
// (src/Algorithms_Create_Fluid_Particle_Depth.h:21-43): an interior cell with
// an empty layer no deeper than the removal depth is refilled too, and every
// interior cell gets layer 0.
// no_particles: the stage form Algorithms_Create_Interior_Depth
// (src/Algorithms_Create_Interior_Depth.h:20-40), which sets the layers (and
// SetFluid on inflow cells) without adding particles.
__global__ void k_refill(const int* __restrict__ blist, const int* __restrict__ bkey, int8_t* lay,
                         const uint8_t* __restrict__ type, const int16_t* __restrict__ depth, double* px,
                         double* py, double* pz, int64_t cap_particles, unsigned long long seed, Params P,
                         Scalars* ds, int no_particles) {
  int n = ds->nlive;
  const int side = 2 * P.refill_cube + 1;
  const int per = P.refill_cube > 0 ? side * side * side : 8;
  const double dh = 1. / side;
  for (int bi = blockIdx.x; bi < n; bi += gridDim.x) {
    int b = blist[bi];
    size_t base = (size_t)b * kCells;
    for (int o = threadIdx.x; o < kCells; o += blockDim.x) {
      const uint8_t t = type[base + o];
      const bool empty = lay[base + o] == kEmpty;
      bool refill = t == MAC_CELL_INFLOW && empty;
      if (P.depth_mode && t == MAC_CELL_INTERIOR) {
        refill = empty && depth[base + o] <= P.depth_remove;
        if (!refill) {
          lay[base + o] = 0;
          continue;
        }
      }
      if (!refill) continue;
      if (no_particles) {
        lay[base + o] = 0;
        continue;
      }
      int kx = bkey[3 * b] * 8 + (o & 7), ky = bkey[3 * b + 1] * 8 + ((o >> 3) & 7),
          kz = bkey[3 * b + 2] * 8 + (o >> 6);
      unsigned long long pos = atomicAdd((unsigned long long*)&ds->np, (unsigned long long)per);
      if ((int64_t)pos + per > cap_particles) {
        atomicOr(&ds->err, kErrParticles);
        atomicAdd((unsigned long long*)&ds->np, (unsigned long long)(-(long long)per));
        continue;
      }
      if (P.refill_cube > 0) {
        const int k[3] = {kx, ky, kz};
        for (int s = 0; s < per; ++s) {
          const int tt[3] = {s % side - P.refill_cube, (s / side) % side - P.refill_cube,
                             s / (side * side) - P.refill_cube};
          double p[3];
          for (int i = 0; i < 3; ++i) p[i] = (k[i] + tt[i] * dh) * P.h[i];
          px[pos + s] = p[0];
          py[pos + s] = p[1];
          pz[pos + s] = p[2];
        }
      } else {
        for (int s = 0; s < 8; ++s) {
          double p[3];
          jitter8(seed, kx, ky, kz, s, P, p);
          px[pos + s] = p[0];
          py[pos + s] = p[1];
          pz[pos + s] = p[2];
        }
      }
      lay[base + o] = 0;
    }
  }
}

// ------------------------------------------------ Update_CellType_Layer
// Bricks near layer-0 cells are created up front (a BFS of LayerMax+1 levels
// stays within ceil((LayerMax+1)/8) bricks); bricks that end with no existing
// cell are freed by the delete pass, exactly as a chunk the reference never
// created.
__global__ void k_dilate(const int* __restrict__ blist, const int* __restrict__ bkey,
                         const int8_t* __restrict__ lay, unsigned long long* hk, const int* hv, int64_t hcap,
                         int* newslots, int64_t cap_new, int R, Scalars* ds) {
  __shared__ int any0;
  int n = ds->nlive;
  for (int bi = blockIdx.x; bi < n; bi += gridDim.x) {
    int b = blist[bi];
    if (threadIdx.x == 0) any0 = 0;
    __syncthreads();
    for (int o = threadIdx.x; o < kCells; o += blockDim.x)
      if (lay[(size_t)b * kCells + o] == 0) any0 = 1;
    __syncthreads();
    if (any0) {
      int side = 2 * R + 1, tot = side * side * side;
      for (int d = threadIdx.x; d < tot; d += blockDim.x) {
        int dx = d % side - R, dy = (d / side) % side - R, dz = d / (side * side) - R;
        if (!dx && !dy && !dz) continue;
        unsigned long long key = pack_key(bkey[3 * b] + dx, bkey[3 * b + 1] + dy, bkey[3 * b + 2] + dz);
        if (hash_find(hk, hv, hcap, key) == -1) hash_insert(hk, hcap, key, newslots, ds, cap_new);
      }
    }
    __syncthreads();
  }
}

__device__ inline int8_t lay_at(const int8_t* __restrict__ lay, const int* __restrict__ nbr, int b, int x, int y,
                                int z) {
  int nb = nb_brick<8>(nbr, b, x, y, z);
  if (nb < 0) return kMissing;
  return lay[(size_t)nb * kCells + slot<8>(wrap<8>(x), wrap<8>(y), wrap<8>(z))];
}

// Level L of the layer BFS (src/Algorithms_Update_CellType_Layer.h:49-72): a
// missing or empty cell with a 6-neighbour of layer L-1 gets layer L and
// SetAir (fluid -> air only, src/Data_CellType_Fluid_Air_Solid_Inflow.tpp:141-148).
// For L = 1 the neighbours of layer 0 are exactly the seeds of :27-48. Cells
// written in this launch change from {-2,-1} to L, never to L-1, so the reads
// of neighbour layers are race-free. ring != 0 runs the final +1-face ring
// (:73-88): only the -e_i neighbours (i.e. the cell is the +e_i face of a
// layer-LayerMax cell) count. SetAir turns fluid and (depth composition)
// interior cells into air
// (src/Data_CellType_Fluid_Air_Solid_Inflow_Interior_0_Pres.tpp:217-223).
__global__ void k_bfs_level(const int* __restrict__ blist, const int* __restrict__ nbr, int8_t* lay,
                            uint8_t* type, int L, int ring, Scalars* ds) {
  int n = ds->nlive;
  for (int bi = blockIdx.x; bi < n; bi += gridDim.x) {
    int b = blist[bi];
    for (int o = threadIdx.x; o < kCells; o += blockDim.x) {
      size_t c = (size_t)b * kCells + o;
      int8_t l = lay[c];
      if (l != kMissing && l != kEmpty) continue;
      int x = o & 7, y = (o >> 3) & 7, z = o >> 6;
      int8_t want = (int8_t)(L - 1);
      // all neighbour layers are loaded before any is compared (no load waits
      // on another's test); a neighbour being set to L by this launch never
      // equals L - 1, so reading its old or new layer is the same
      const int8_t lm[3] = {lay_at(lay, nbr, b, x - 1, y, z), lay_at(lay, nbr, b, x, y - 1, z),
                            lay_at(lay, nbr, b, x, y, z - 1)};
      int8_t lp[3] = {kMissing, kMissing, kMissing};
      if (!ring) {
        lp[0] = lay_at(lay, nbr, b, x + 1, y, z);
        lp[1] = lay_at(lay, nbr, b, x, y + 1, z);
        lp[2] = lay_at(lay, nbr, b, x, y, z + 1);
      }
      bool hit = lm[0] == want || lm[1] == want || lm[2] == want;
      if (!ring && !hit) hit = lp[0] == want || lp[1] == want || lp[2] == want;
      if (hit) {
        lay[c] = (int8_t)L;
        const uint8_t t = type[c];
        if (t == MAC_CELL_FLUID || t == MAC_CELL_INTERIOR) type[c] = MAC_CELL_AIR;
      }
    }
  }
}

// ------------------------------------- Update_CellType_Layer_Depth: depth
// src/Algorithms_Update_CellType_Layer_Depth.h:33-55: every existing cell's
// depth is emptied, and a layer-0 cell with a missing or empty-layer face
// neighbour (read before the air layers are added) gets depth 0 and seeds the
// inward BFS of :104-134.
__global__ void k_depth_seed(const int* __restrict__ blist, const int* __restrict__ nbr,
                             const int8_t* __restrict__ lay, int16_t* depth, Scalars* ds) {
  int n = ds->nlive;
  for (int bi = blockIdx.x; bi < n; bi += gridDim.x) {
    int b = blist[bi];
    for (int o = threadIdx.x; o < kCells; o += blockDim.x) {
      size_t c = (size_t)b * kCells + o;
      int8_t l = lay[c];
      if (l == kMissing) continue;
      int16_t d = -1;
      if (l == 0) {
        int x = o & 7, y = (o >> 3) & 7, z = o >> 6;
        const int8_t nl[6] = {lay_at(lay, nbr, b, x - 1, y, z), lay_at(lay, nbr, b, x + 1, y, z),
                              lay_at(lay, nbr, b, x, y - 1, z), lay_at(lay, nbr, b, x, y + 1, z),
                              lay_at(lay, nbr, b, x, y, z - 1), lay_at(lay, nbr, b, x, y, z + 1)};
        for (int f = 0; f < 6; ++f)
          if (nl[f] == kMissing || nl[f] == kEmpty) d = 0;
      }
      depth[c] = d;
    }
  }
}

// The inward BFS of src/Algorithms_Update_CellType_Layer_Depth.h:104-134 as a
// min-plus relaxation, which reaches the same fixed point (the BFS distance
// through face-adjacent layer-0 cells from the depth-0 seeds) in any order:
// each block takes one brick with a one-cell halo into shared memory and
// relaxes d(c) = min(d(c), d(n) + 1) over its layer-0 cells until nothing
// changes, then writes the lowered depths back. Halo values read while a
// neighbouring brick is being relaxed are older upper bounds, so the host
// repeats the launch until no depth changes (about max depth / 8 launches).
// Unreached layer-0 cells keep -1, as in the reference.
constexpr int16_t kDepthInf = 0x7fff;
constexpr int16_t kDepthNone = -2;

__global__ void __launch_bounds__(512) k_depth_relax(const int* __restrict__ blist, const int* __restrict__ nbr,
                                                     const int8_t* __restrict__ lay, int16_t* depth, Scalars* ds) {
  __shared__ int16_t sd[1000];  // 10^3 with halo: kDepthNone off the layer-0 set, kDepthInf unreached
  int n = ds->nlive;
  const int t = threadIdx.x;
  const int x = t & 7, y = (t >> 3) & 7, z = t >> 6;
  const int me = (x + 1) + 10 * ((y + 1) + 10 * (z + 1));
  for (int bi = blockIdx.x; bi < n; bi += gridDim.x) {
    const int b = blist[bi];
    for (int i = t; i < 1000; i += blockDim.x) {
      const int hx = i % 10 - 1, hy = (i / 10) % 10 - 1, hz = i / 100 - 1;
      const int nb = nb_brick<8>(nbr, b, hx, hy, hz);
      int16_t v = kDepthNone;
      if (nb >= 0) {
        const size_t c = (size_t)nb * kCells + slot<8>(wrap<8>(hx), wrap<8>(hy), wrap<8>(hz));
        if (lay[c] == 0) {
          const int16_t d = depth[c];
          v = d < 0 ? kDepthInf : d;
        }
      }
      sd[i] = v;
    }
    __syncthreads();
    const int16_t start = sd[me];
    const bool part = start != kDepthNone && start != 0;  // relaxed: layer-0 non-seed cells
    int16_t cur = start;
    while (true) {
      bool ch = false;
      if (part) {
        int16_t m = kDepthInf;
        const int nn[6] = {me - 1, me + 1, me - 10, me + 10, me - 100, me + 100};
        for (int f = 0; f < 6; ++f) {
          const int16_t v = sd[nn[f]];
          if (v >= 0 && v < m) m = v;
        }
        if (m < kDepthInf - 1 && m + 1 < cur) {
          cur = (int16_t)(m + 1);
          sd[me] = cur;
          ch = true;
        }
      }
      if (!__syncthreads_or(ch)) break;
    }
    if (part && cur < start) {
      depth[(size_t)b * kCells + t] = cur;
      ds->dchanged = 1;
    }
    __syncthreads();
  }
}

__global__ void k_depth_flag_clear(Scalars* ds) { ds->dchanged = 0; }

// Materials of :117-124: a layer-0 cell reached at depth d >= 1 becomes fluid
// (SetFluid: from air or interior) when d < DepthInterior and interior
// (SetInterior: always) otherwise; the seeds keep their material.
__global__ void k_depth_types(const int* __restrict__ blist, const int8_t* __restrict__ lay,
                              const int16_t* __restrict__ depth, uint8_t* type, Params P, Scalars* ds) {
  int n = ds->nlive;
  for (int bi = blockIdx.x; bi < n; bi += gridDim.x) {
    size_t base = (size_t)blist[bi] * kCells;
    for (int o = threadIdx.x; o < kCells; o += blockDim.x) {
      size_t c = base + o;
      if (lay[c] != 0) continue;
      int16_t d = depth[c];
      if (d < 1) continue;
      uint8_t t = type[c];
      if (d < P.depth_interior) {
        if (t == MAC_CELL_AIR || t == MAC_CELL_INTERIOR) type[c] = MAC_CELL_FLUID;
      } else {
        type[c] = MAC_CELL_INTERIOR;
      }
    }
  }
}

// ------------------------------------------------------ Delete_MacCell
// src/Algorithms_Delete_MacCell.h:22-44: existing cells with an empty layer
// and no no-delete mark are erased; a brick left without cells is freed
// (src/ChunkHashTable.tpp:132-147).
__global__ void k_delete(const int* __restrict__ blist, int8_t* lay, const uint8_t* __restrict__ flags,
                         uint8_t* alive, Scalars* ds) {
  __shared__ int any;
  int n = ds->nlive;
  for (int bi = blockIdx.x; bi < n; bi += gridDim.x) {
    int b = blist[bi];
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    size_t base = (size_t)b * kCells;
    int mine = 0;
    for (int o = threadIdx.x; o < kCells; o += blockDim.x) {
      int8_t l = lay[base + o];
      if (l == kEmpty && !(flags[base + o] & MAC_FLAG_NODELETE)) {
        lay[base + o] = kMissing;
        l = kMissing;
      }
      mine |= (l != kMissing);
    }
    if (mine) any = 1;
    __syncthreads();
    if (threadIdx.x == 0) alive[b] = (uint8_t)any;
    __syncthreads();
  }
}

__global__ void k_compact(const int* __restrict__ blist, int* blist2, int* freelist, const uint8_t* alive,
                          Scalars* ds) {
  int n = ds->nlive;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int b = blist[i];
    if (alive[b]) blist2[atomicAdd(&ds->nlive_new, 1)] = b;
    else freelist[atomicAdd(&ds->nfree, 1)] = b;
  }
}

__global__ void k_compact_done(Scalars* ds) {
  ds->nlive = ds->nlive_new;
  ds->nlive_new = 0;
}

// ------------------------------------------------ Calculate_Time_Step
// src/Algorithms_Calculate_Time_Step.h:41-62: max over fluid cells of
// sum_i (u_i * (1/h_i))^2 (pow(x,2) is x*x), then dt = 1/sqrt(max)*factor and
// Policy_CheckDT's clamp (src/Policy_CheckDT.h:16-29). The same pass counts
// fluid cells for the throughput metric.
__global__ void k_cfl(const int* __restrict__ blist, const int8_t* __restrict__ lay,
                      const uint8_t* __restrict__ type, const double* __restrict__ ux,
                      const double* __restrict__ uy, const double* __restrict__ uz, Params P, Scalars* ds) {
  __shared__ unsigned long long smax;
  __shared__ int scount;
  int n = ds->nlive;
  double mx = 0;
  int cnt = 0;
  for (int bi = blockIdx.x; bi < n; bi += gridDim.x) {
    size_t base = (size_t)blist[bi] * kCells;
    for (int o = threadIdx.x; o < kCells; o += blockDim.x) {
      size_t c = base + o;
      if (lay[c] == kMissing || !is_fluid(type[c])) continue;
      ++cnt;
      double t = 0;
      double v = ux[c] * P.ih[0];
      t += v * v;
      v = uy[c] * P.ih[1];
      t += v * v;
      v = uz[c] * P.ih[2];
      t += v * v;
      if (t > mx) mx = t;
    }
  }
  if (threadIdx.x == 0) {
    smax = 0;
    scount = 0;
  }
  __syncthreads();
  atomicMax(&smax, (unsigned long long)__double_as_longlong(mx));
  atomicAdd(&scount, cnt);
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicMax(&ds->cfl_bits, smax);
    atomicAdd((unsigned long long*)&ds->nfluid, (unsigned long long)scount);
  }
}

__global__ void k_cfl_reset(Scalars* ds) {
  ds->cfl_bits = 0;
  ds->nfluid = 0;
}

__global__ void k_dt_finalize(Params P, Scalars* ds) {
  double mx = __longlong_as_double((long long)ds->cfl_bits);
  double dt = 1 / sqrt(mx) * P.cfl;
  if (dt < P.dt_min) dt = P.dt_min;
  else if (dt > P.dt_max) dt = P.dt_max;
  ds->dt = dt;
}

// ------------------------------------------------------------ drivers
int rebuild_index(Ctx* c) {
  cudaStream_t st = c->stream;
  k_hash_clear<<<grid_for(c->hcap, 256), 256, 0, st>>>(c->hkeys, c->hval, c->hcap); MAC_COUNT(c);
  k_hash_insert_live<<<kTopoBlocks, 256, 0, st>>>(c->blist, c->bkey, c->hkeys, c->hval, c->hcap, c->ds); MAC_COUNT(c);
  k_build_nbr<<<kTopoBlocks, 256, 0, st>>>(c->blist, c->bkey, c->hkeys, c->hval, c->hcap, c->nbr, c->ds); MAC_COUNT(c);
  c->system_ready = false;
  return check(cudaGetLastError());
}

static void alloc_new(Ctx* c) {
  cudaStream_t st = c->stream;
  k_alloc_bricks<<<kTopoBlocks, 256, 0, st>>>(c->newslots, c->hkeys, c->hval, c->bkey, c->blist, c->freelist,
                                               c->lay, c->type, c->flags, c->f64, c->depth, c->u2,
                                               (size_t)c->cap_bricks * kCells, c->cap_bricks, c->ds); MAC_COUNT(c);
}

int topo_initialize(Ctx* c) {
  k_initialize<<<kTopoBlocks, 256, 0, c->stream>>>(c->blist, c->lay, c->type, c->dp.depth_mode ? c->depth : nullptr,
                                                   c->ds); MAC_COUNT(c);
  return check(cudaGetLastError());
}

int topo_layer_initial(Ctx* c) {
  cudaStream_t st = c->stream;
  int g = kTopoBlocks * 2;
  k_clear_note<<<1, 1, 0, st>>>(c->ds); MAC_COUNT(c);
  uint8_t* keep = c->dp.depth_mode ? c->pkeep : nullptr;
  // the position the topology reads (Data_Particle::imove_particle): 0, or 2
  // during pipeline B's stages 2-4
  const double* kx = c->imove == 2 ? c->pbuf[1][0] : c->px;
  const double* ky = c->imove == 2 ? c->pbuf[1][1] : c->py;
  const double* kz = c->imove == 2 ? c->pbuf[1][2] : c->pz;
  k_mark_particles<<<g, 256, 0, st>>>(kx, ky, kz, c->dp, c->hkeys, c->hval, c->hcap, c->newslots,
                                      c->cap_bricks, c->lay, c->type, c->depth, keep, c->ds, 0); MAC_COUNT(c);
  k_note_missing<<<1, 1, 0, st>>>(c->ds); MAC_COUNT(c);
  alloc_new(c);
  k_after_alloc<<<1, 1, 0, st>>>(c->ds); MAC_COUNT(c);
  k_mark_particles<<<g, 256, 0, st>>>(kx, ky, kz, c->dp, c->hkeys, c->hval, c->hcap, c->newslots,
                                      c->cap_bricks, c->lay, c->type, c->depth, keep, c->ds, 1); MAC_COUNT(c);
  k_clear_note<<<1, 1, 0, st>>>(c->ds); MAC_COUNT(c);
  if (keep) {
    PartMove M;
    M.src[0] = c->px; M.src[1] = c->py; M.src[2] = c->pz;
    M.dst[0] = c->px2; M.dst[1] = c->py2; M.dst[2] = c->pz2;
    M.n = 3;
    if (c->dp.pipeline == 1) {
      for (int k = 0; k < 2; ++k)
        for (int i = 0; i < 3; ++i) {
          M.src[3 + 3 * k + i] = c->pbuf[k][i];
          M.dst[3 + 3 * k + i] = c->pbuf2[k][i];
        }
      M.n = 9;
    }
    k_compact_particles<<<g, 256, 0, st>>>(M, keep, c->ds); MAC_COUNT(c);
    k_compact_particles_done<<<1, 1, 0, st>>>(c->ds); MAC_COUNT(c);
    std::swap(c->px, c->px2);
    std::swap(c->py, c->py2);
    std::swap(c->pz, c->pz2);
    if (c->dp.pipeline == 1)
      for (int k = 0; k < 2; ++k)
        for (int i = 0; i < 3; ++i) std::swap(c->pbuf[k][i], c->pbuf2[k][i]);
  }
  c->system_ready = false;
  return check(cudaGetLastError());
}

int topo_create_fluid(Ctx* c) {
  k_refill<<<kTopoBlocks, 256, 0, c->stream>>>(c->blist, c->bkey, c->lay, c->type, c->depth, c->px, c->py, c->pz,
                                                c->cap_particles, (unsigned long long)c->seed, c->dp, c->ds, 0); MAC_COUNT(c);
  return check(cudaGetLastError());
}

// Relaxation launches until no depth changes; each launch carries the front at
// least one brick further, so the bound below (the pool's brick count) is
// never reached by a valid world.
static int depth_bfs(Ctx* c) {
  cudaStream_t st = c->stream;
  const int limit = (int)(c->cap_bricks < 1000000 ? c->cap_bricks : 1000000) + 2;
  for (int it = 0;; ++it) {
    if (it >= limit) return MAC_ERR_TIMEOUT;
    k_depth_flag_clear<<<1, 1, 0, st>>>(c->ds); MAC_COUNT(c);
    k_depth_relax<<<kTopoBlocks, 512, 0, st>>>(c->blist, c->nbr, c->lay, c->depth, c->ds); MAC_COUNT(c);
    int rc = read_scalars(c);
    if (rc) return rc;
    if (!c->hs->dchanged) break;
  }
  k_depth_types<<<kTopoBlocks, 256, 0, st>>>(c->blist, c->lay, c->depth, c->type, c->dp, c->ds); MAC_COUNT(c);
  return check(cudaGetLastError());
}

int topo_update_layer(Ctx* c) {
  cudaStream_t st = c->stream;
  int R = (c->dp.layer_max + 1 + 7) / 8;
  if (R < 1) R = 1;
  k_dilate<<<kTopoBlocks, 256, 0, st>>>(c->blist, c->bkey, c->lay, c->hkeys, c->hval, c->hcap, c->newslots,
                                         c->cap_bricks, R, c->ds); MAC_COUNT(c);
  alloc_new(c);
  k_after_alloc<<<1, 1, 0, st>>>(c->ds); MAC_COUNT(c);
  k_build_nbr<<<kTopoBlocks, 256, 0, st>>>(c->blist, c->bkey, c->hkeys, c->hval, c->hcap, c->nbr, c->ds); MAC_COUNT(c);
  if (c->dp.depth_mode) {
    k_depth_seed<<<kTopoBlocks, 256, 0, st>>>(c->blist, c->nbr, c->lay, c->depth, c->ds); MAC_COUNT(c);
  }
  for (int L = 1; L <= c->dp.layer_max; ++L) {
    k_bfs_level<<<kTopoBlocks, 256, 0, st>>>(c->blist, c->nbr, c->lay, c->type, L, 0, c->ds); MAC_COUNT(c);
  }
  k_bfs_level<<<kTopoBlocks, 256, 0, st>>>(c->blist, c->nbr, c->lay, c->type, c->dp.layer_max + 1, 1, c->ds); MAC_COUNT(c);
  c->system_ready = false;
  if (c->dp.depth_mode) {
    int rc = depth_bfs(c);
    if (rc) return rc;
  }
  return check(cudaGetLastError());
}

int topo_delete(Ctx* c) {
  cudaStream_t st = c->stream;
  k_delete<<<kTopoBlocks, 256, 0, st>>>(c->blist, c->lay, c->flags, c->alive, c->ds); MAC_COUNT(c);
  k_compact<<<kTopoBlocks, 256, 0, st>>>(c->blist, c->blist2, c->freelist, c->alive, c->ds); MAC_COUNT(c);
  k_compact_done<<<1, 1, 0, st>>>(c->ds); MAC_COUNT(c);
  int* t = c->blist;
  c->blist = c->blist2;
  c->blist2 = t;
  c->system_ready = false;
  return rebuild_index(c);
}

int topo_dt(Ctx* c) {
  cudaStream_t st = c->stream;
  size_t cap = (size_t)c->cap_bricks * kCells;
  k_cfl_reset<<<1, 1, 0, st>>>(c->ds); MAC_COUNT(c);
  k_cfl<<<kTopoBlocks, 256, 0, st>>>(c->blist, c->lay, c->type, c->f64 + U0X * cap, c->f64 + U0Y * cap,
                                      c->f64 + U0Z * cap, c->dp, c->ds); MAC_COUNT(c);
  k_dt_finalize<<<1, 1, 0, st>>>(c->dp, c->ds); MAC_COUNT(c);
  return check(cudaGetLastError());
}

int topo_finish(Ctx* c) {
  int rc = read_scalars(c);
  c->stats.fluid_cells = c->hs->nfluid;
  return rc;
}

// init2 of pipeline B's stages (test/Jet3.cpp:549): the depth topology with
// Create_Interior_Depth and no time step, at the current particle buffer.
int topology_stage(Ctx* c) {
  int rc;
  prof_begin(c, PH_TOPOLOGY);
  if ((rc = topo_initialize(c))) return rc;
  if ((rc = topo_layer_initial(c))) return rc;
  k_refill<<<kTopoBlocks, 256, 0, c->stream>>>(c->blist, c->bkey, c->lay, c->type, c->depth, c->px, c->py, c->pz,
                                                c->cap_particles, (unsigned long long)c->seed, c->dp, c->ds, 1); MAC_COUNT(c);
  if ((rc = topo_update_layer(c))) return rc;
  if ((rc = topo_delete(c))) return rc;
  prof_end(c, PH_TOPOLOGY);
  return read_scalars(c);  // live bricks and particles; the fluid count stays the step's
}

int topology_rebuild(Ctx* c, bool first_init_order) {
  int rc;
  if (!first_init_order) ++c->seed;
  prof_begin(c, PH_TOPOLOGY);
  if ((rc = topo_initialize(c))) return rc;
  if (first_init_order) {
    if ((rc = topo_create_fluid(c))) return rc;
    if ((rc = topo_layer_initial(c))) return rc;
  } else {
    if ((rc = topo_layer_initial(c))) return rc;
    if ((rc = topo_create_fluid(c))) return rc;
  }
  if ((rc = topo_update_layer(c))) return rc;
  if ((rc = topo_delete(c))) return rc;
  if (!first_init_order)
    if ((rc = topo_dt(c))) return rc;
  prof_end(c, PH_TOPOLOGY);
  return topo_finish(c);
}

}  // namespace mac
