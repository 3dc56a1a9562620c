// Device-side data model of the brick grid and the context shared by the kernels.
//
// The reference's sparse chunk grid (src/ChunkHashTable.h:22-160: an
// unordered_map from chunk key to an 8^3 chunk of SoA arrays with an existence
// bitset) becomes:
//   * a pool of bricks; brick b owns cells [b*512, b*512+512), slot x+8y+64z,
//   * an open-addressing hash table from packed brick key to pool index,
//     rebuilt after every topology pass,
//   * a compact list of live bricks and a free list,
//   * a 27-entry neighbour table per live brick (the reference links chunks to
//     their 2*DIM neighbours: src/Hook_Neighbour_List_key.h:97-120).
// Per-cell fields are SoA arrays over the pool. Existence and layer share one
// signed byte `lay`: -2 = cell does not exist, -1 = exists with an empty layer,
// >= 0 = layer. The reference keeps a separate bit and leaves the layer of an
// erased cell stale; that stale layer is never read before it is rewritten
// (every re-creation path sets the layer), so folding the two is exact and lets
// one byte store publish both at once.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/mac_gpu.h"

namespace mac {

constexpr int kBrick = 8;
constexpr int kCells = 512;
constexpr int kNbr = 27;
constexpr int kSelf = 13;
constexpr int8_t kMissing = -2;
constexpr int8_t kEmpty = -1;
constexpr uint64_t kEmptyKey = ~0ull;
constexpr int32_t kPending = -2;
constexpr int kLevels = 4;  // brick-local multigrid levels: 8^3, 4^3, 2^3, 1 cell per brick

enum ErrBits : int {
  kErrBricks = 1,
  kErrParticles = 2,
  kErrHash = 4,
  kErrPending = 8,
  kErrTimeout = 16,  // a bounded wait on an asynchronous copy ran out
};

// Field indices of the FP64 per-cell block.
enum F64 : int { U0X = 0, U0Y, U0Z, U1X, U1Y, U1Z, AX, AY, AZ, PRES, NF64 };

struct Scalars {
  int32_t nlive;
  int32_t nlive_new;
  int32_t nfree;
  int32_t nnew;       // newly inserted hash slots waiting for a brick
  int32_t npending;   // particles waiting for their brick
  int32_t err;
  int64_t np;
  double dt;
  double t;
  unsigned long long cfl_bits;  // max over fluid cells of sum (u_i/h_i)^2, as ordered bits
  unsigned long long div_bits;  // max |div| after a projection, as ordered bits
  int64_t nfluid;
  int64_t nunknown;
  // CG scalars
  double rz, rz_new, pq, rr, bnorm2, alpha, beta;
  int32_t done;
  int32_t iters;
  int32_t bbox[6];    // brick key bounds of the domain bricks (min xyz, max xyz)
  int32_t ndom;       // bricks holding an in-domain cell
  int32_t pad_;
  unsigned long long bad_reads;  // particles whose stencil touched a missing cell
  unsigned long long np_new;     // particle count after the removal pass (depth composition)
  int32_t dchanged;              // a depth relaxation launch lowered some depth
  int32_t pad2_;
};

// Phases timed with CUDA events when profiling is on (mac_set_profiling);
// the order matches MAC_PHASE_* in include/mac_gpu.h.
enum Phase : int {
  PH_TOPOLOGY = 0,
  PH_FORCES,
  PH_SETUP,
  PH_DIVERGENCE,
  PH_SPMV,
  PH_CGVEC,
  PH_VCYCLE,
  PH_GRADIENT,
  PH_EXTRAPOLATE,
  PH_MOVE,
  kPhases
};

struct Params {
  double h[3], ih[3], ih2[3];
  double cfl, dt_min, dt_max, g;
  int gaxis;     // 0..2
  int layer_max;
  int interp_sym;
  // viscosity (0: inviscid composition) and pow(1/h, 2) as the Laplacian of
  // src/Policy_Laplacian_Speed.h:22-36 computes it
  double nu, lih2[3];
  // depth composition (Policy_Depth) and the refill policy (0: jitter8, n: cube(n))
  int depth_mode, depth_interior, depth_remove, refill_cube;
  int pipeline;  // 0: pipeline A (RK2-TVD + particle RK4); 1: pipeline B (Algorithms_RungeKutta_all)
  // inverse diagonal of the level-0 operator by active faces per axis
  // (index ax + 3 ay + 9 az, each 0..2); 0 when no face is active
  double dtab[27];
  // multigrid smoother: weights of the two Jacobi sweeps before and after each
  // coarse correction, and of the single sweep of the one-sweep finest level
  double mgw1, mgw2, mgws;
};

// Dense grid over the bounding box of the domain bricks (one cell per brick).
struct DenseGrid {
  int x0, y0, z0, nx, ny, nz;
  __host__ __device__ int64_t index(int bx, int by, int bz) const {
    return (int64_t)(bx - x0) + (int64_t)nx * ((int64_t)(by - y0) + (int64_t)ny * (bz - z0));
  }
  __host__ __device__ bool contains(int bx, int by, int bz) const {
    return (unsigned)(bx - x0) < (unsigned)nx && (unsigned)(by - y0) < (unsigned)ny && (unsigned)(bz - z0) < (unsigned)nz;
  }
  // index of a brick's dense cell; 0 for a brick outside the box (a live
  // brick without in-domain cells next to a domain brick: its value is read
  // but enters nothing, since the face weight to it is zero)
  __host__ __device__ int64_t index_or0(int bx, int by, int bz) const {
    return contains(bx, by, bz) ? index(bx, by, bz) : 0;
  }
};

constexpr int kMaxDense = 12;
struct DenseDesc {
  int nx, ny, nz;
  int64_t n, off;
};

struct Ctx {
  mac_params prm;
  Params dp;
  cudaStream_t stream = nullptr;
  int64_t cap_bricks = 0, cap_particles = 0, hcap = 0, cap_pending = 0;
  uint64_t seed = 0;
  int own_device = 0;

  // brick pool
  int* bkey = nullptr;        // [cap][3]
  int8_t* lay = nullptr;      // [cap*512]
  uint8_t* type = nullptr;    // [cap*512]
  uint8_t* flags = nullptr;   // [cap*512]
  double* f64 = nullptr;      // [NF64][cap*512]
  double* pdir = nullptr;     // [cap*512] Dirichlet air pressure, NaN off the boundary (viscous only)
  int16_t* depth = nullptr;   // [cap*512] distance to the surface, -1 empty (depth composition only)
  uint8_t* pkeep = nullptr;   // [max_particles] removal marks of the particle pass (depth composition only)
  // pipeline B (Algorithms_RungeKutta_all): speed buffer 2, particle positions
  // 1 and 2 with their compaction scratch, and the position the topology reads
  double* u2 = nullptr;       // [3][cap*512]
  double* pbuf[2][3] = {};    // [max_particles] each
  double* pbuf2[2][3] = {};
  int imove = 0;              // 0 or 2 (Data_Particle::imove_particle)
  int* nbr = nullptr;         // [cap][27]
  int* blist = nullptr;       // live bricks (current)
  int* blist2 = nullptr;      // scratch for compaction
  int* freelist = nullptr;
  uint8_t* alive = nullptr;   // [cap] per-brick flag
  // hash
  unsigned long long* hkeys = nullptr;
  int* hval = nullptr;
  int* newslots = nullptr;    // [cap]
  // particles (SoA)
  double* px = nullptr;
  double* py = nullptr;
  double* pz = nullptr;
  int64_t* pending = nullptr; // particle indices waiting for a brick
  double* px2 = nullptr;      // binned copy (swapped with px each move)
  double* py2 = nullptr;
  double* pz2 = nullptr;
  int* pbrick = nullptr;      // 512 * brick + cell of each particle's cell (brick cap: no brick)
  int* bcount = nullptr;      // [cap+1] particles per brick (last: no brick)
  uint32_t* lmask = nullptr;  // [cap] per live brick: bit l set when a cell has layer l (l >= 31 on bit 31)
  int* bcursor = nullptr;     // [(cap+1)*512] particles per (brick, cell), then each cell's running slot
  int64_t* boff = nullptr;    // [cap+2] bin offsets
  // pressure system and solver
  uint16_t* fmask = nullptr;  // [cap*512] face classes of the level-0 operator
  double* x = nullptr;        // solution (pressure in domain)
  double* b = nullptr;        // right-hand side
  double* r = nullptr;
  double* r2 = nullptr;       // the residual's second buffer: a V-cycle that finishes the
                              // previous CG iteration writes the new r there
  double* z = nullptr;
  double* pd = nullptr;       // search direction
  double* pd2 = nullptr;      // its previous value (the update reads neighbours' old p)
  double* q = nullptr;
  double* partial = nullptr;  // per-block partial sums
  int64_t npartial = 0;
  // multigrid (T = double or float storage, chosen by the solver)
  void* mg_e[kLevels] = {};   // correction
  void* mg_e2[kLevels] = {};  // ping-pong
  void* mg_r[kLevels] = {};   // level residual (levels >= 1)
  void* mg_w[kLevels] = {};   // [4][cells]: left-face weights x,y,z and Dirichlet diagonal
  void* mg_dinv[kLevels] = {};
  int mg_float = 0;
  double mg_scale = 0.6;      // coarse-operator scale of the Galerkin products
  int mg_sweeps0 = 2;         // Jacobi sweeps before and after the coarse correction at level 0 (1 or 2)
  int mg_bulk = 0;            // 1: the V-cycle's first kernel prefetches bricks with cp.async.bulk
  int bulk_grid = 0;          // its grid (blocks resident on all SMs at once)
  int npart_head = 0;         // partial sums the V-cycle's first kernel left (its grid)
  // learned preconditioner (flexible CG): the network and the previous z
  void* unet = nullptr;
  double* zold = nullptr;
  double learned_omega = 0.8;
  int* dbl = nullptr;          // bricks holding an in-domain cell, by brick coordinates (x fastest)
  int* drow = nullptr;         // per domain brick: pool index and six face neighbours (8 ints)
  int ndom_host = 0;
  int* dbl_map = nullptr;      // ordering scratch: one slot per brick of the domain's bounding box
  int64_t dbl_map_n = 0;
  int* dbl_cnt = nullptr;      // ordering scratch: per-block counts, then offsets
  DenseGrid g3{};
  DenseDesc dense[kMaxDense] = {};
  int ndense = 0;
  void* dense_buf = nullptr;   // dense levels: 9 arrays (e, e2, r, 6 weights) per cell
  size_t dense_bytes = 0;
  size_t dense_smem = 0;
  int dense_lo = 1;              // first dense level of the one-block coarse solve
  int blk_max_cells = 1024;      // the largest level it takes; larger ones run device-wide
  double* coarse_inv = nullptr;  // [64][64] inverse of the coarsest dense level
  int* coarse_ok = nullptr;      // 1 when coarse_inv is valid
  int smem_optin = 0;
  // scalars
  Scalars* ds = nullptr;      // device
  Scalars* hs = nullptr;      // pinned host mirror
  Scalars* hs_lag = nullptr;  // [2] pinned: the scalars after the last two CG iterations
  cudaEvent_t ev_lag[2] = {};
  int nlive_host = 0;
  int64_t np_host = 0;
  mac_stats stats{};
  bool system_ready = false;
  // drop-in CSC solver
  int csc_n = 0;
  int* csc_off = nullptr;
  int* csc_ind = nullptr;
  double* csc_val = nullptr;
  double* csc_vec = nullptr;   // [7][n] + scalars (CG), [11][n] + scalars (BiCGStab)
  int csc_general = 0;         // 1: not the symmetric negative-diagonal form, solved by BiCGStab
  int* csr_off = nullptr;      // row-major copy for BiCGStab
  int* csr_ind = nullptr;
  double* csr_val = nullptr;
  int* eb_work = nullptr;      // boundary-condition extrapolation: colour counts and cursors
  long long launches = 0;      // kernels launched by this context
  struct Prof* prof = nullptr; // per-phase event timing (null when off)
  int pdl = 1;                 // CG-loop kernels launched with programmatic stream serialisation
  // particle binning on a second stream, overlapping the step's first
  // projection (measured no faster on the 256x256x512 jet: off by default)
  int bin_side = 0;
  int bin_pending = 0;   // the step wants its binning started beside the first solve
  int bin_launched = 0;  // it was: the context's stream must wait on ev_bins
  cudaStream_t side = nullptr;
  cudaEvent_t ev_topo = nullptr;  // the topology is done (the binning may start)
  cudaEvent_t ev_bins = nullptr;  // the binning is done (the move may start)
};

void prof_begin(Ctx* c, int phase);
void prof_end(Ctx* c, int phase);

// Every kernel launch is followed by MAC_COUNT(c) so the context can report
// how many of its kernels ran (mac_launch_count).
#define MAC_COUNT(ctx) (++(ctx)->launches)

// ------------------------------------------------- programmatic dependent launch
// The CG loop runs some twenty dependent kernels per iteration, many of them a
// few microseconds long, so the gap between two of them (the next grid's
// launch and its blocks' ramp-up after the previous grid's last block) is a
// large part of the iteration. Launched with programmatic stream
// serialisation, a kernel's blocks may be scheduled once every block of the
// previous kernel has started (pdl_entry's trigger), and they wait in
// griddepcontrol.wait until that kernel has completed and its writes are
// visible. A kernel launched this way calls pdl_entry() as its first
// statement, on every path: it reads nothing before the wait, and since each
// kernel of the chain waits for its predecessor's completion before it can
// complete itself, completion stays ordered along the whole stream. The wait
// ends because the previous grid depends on nothing that comes after it.
// Without the launch attribute both instructions do nothing.
__device__ __forceinline__ void pdl_entry() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
// A kernel's prologue before pdl_entry() may load what the previous kernel
// does not write: the launch order makes a kernel start only after every
// block of the previous kernel has passed its own wait, i.e. after the kernel
// before that has completed. So the prologue may read static data (brick
// tables, face masks, multigrid weights) and whatever the kernels two or more
// launches back wrote; it writes nothing to global memory, and every thread
// reaches pdl_entry() before it may return.

template <class... P, class... A>
inline void launch_k(const Ctx* c, void (*k)(P...), dim3 grid, dim3 block, size_t smem, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = c->stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = c->pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, k, static_cast<A&&>(args)...);
}

// ---------------------------------------------------------------- helpers
__host__ __device__ inline unsigned long long pack_key(int x, int y, int z) {
  return ((unsigned long long)((uint32_t)(x + (1 << 20)) & 0x1FFFFFu)) |
         ((unsigned long long)((uint32_t)(y + (1 << 20)) & 0x1FFFFFu) << 21) |
         ((unsigned long long)((uint32_t)(z + (1 << 20)) & 0x1FFFFFu) << 42);
}
__host__ __device__ inline void unpack_key(unsigned long long k, int* x, int* y, int* z) {
  *x = (int)(k & 0x1FFFFFu) - (1 << 20);
  *y = (int)((k >> 21) & 0x1FFFFFu) - (1 << 20);
  *z = (int)((k >> 42) & 0x1FFFFFu) - (1 << 20);
}
__host__ __device__ inline unsigned long long hmix(unsigned long long k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  k ^= k >> 33;
  return k;
}
// Floor division by the brick edge (src/ChunkHashTable.tpp:180-196).
__host__ __device__ inline int fdiv8(int v) { return v >= 0 ? v >> 3 : -((-v + 7) >> 3); }

__device__ inline int hash_find(const unsigned long long* __restrict__ hk, const int* __restrict__ hv,
                                int64_t hcap, unsigned long long key) {
  unsigned long long s = hmix(key) & (unsigned long long)(hcap - 1);
  for (int64_t probe = 0; probe < hcap; ++probe) {
    unsigned long long k = hk[s];
    if (k == key) return hv[s];
    if (k == kEmptyKey) return -1;
    s = (s + 1) & (unsigned long long)(hcap - 1);
  }
  return -1;
}

// Neighbour table index of brick offset (dx,dy,dz) in {-1,0,1}^3.
__host__ __device__ inline int nbr_index(int dx, int dy, int dz) { return (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1); }

// Cell (brick, slot) of the cell at local coordinates (x,y,z) of brick `b`
// where the coordinates may leave [0,D) by at most D (one brick). Returns -1
// brick when the neighbour brick is not live.
template <int D>
__device__ inline int nb_brick(const int* __restrict__ nbr, int b, int x, int y, int z) {
  int dx = x < 0 ? -1 : (x >= D ? 1 : 0);
  int dy = y < 0 ? -1 : (y >= D ? 1 : 0);
  int dz = z < 0 ? -1 : (z >= D ? 1 : 0);
  if ((dx | dy | dz) == 0) return b;
  return nbr[(size_t)b * kNbr + nbr_index(dx, dy, dz)];
}
template <int D>
__device__ inline int wrap(int v) { return v < 0 ? v + D : (v >= D ? v - D : v); }
template <int D>
__device__ inline int slot(int x, int y, int z) { return x + D * y + D * D * z; }

// GetIsFluid: fluid, inflow and (depth composition) interior cells
// (src/Data_CellType_Fluid_Air_Solid_Inflow_Interior_0_Pres.tpp:24-44).
__device__ inline bool is_fluid(uint8_t t) {
  return t == MAC_CELL_FLUID || t == MAC_CELL_INFLOW || t == MAC_CELL_INTERIOR;
}

// Ordered-bits max for non-negative doubles.
__device__ inline void atomic_max_nonneg(unsigned long long* a, double v) {
  atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

// Level-0 face classes of an in-domain cell: bit f (f = 2*axis + (sign > 0))
// = interior coupling, bit 8+f = face counts in the diagonal, bit 15 = in domain.
constexpr uint16_t kDomainBit = 0x8000;

// Inverse-diagonal table index from the face classes: active faces on x + 3*(y) + 9*(z).
__device__ inline int active_index(uint16_t m) {
  return __popc((m >> 8) & 3u) + 3 * __popc((m >> 10) & 3u) + 9 * __popc((m >> 12) & 3u);
}

// Cell-index bases of the six face-neighbour bricks of brick b (x-, x+, y-,
// y+, z-, z+), -1 when absent; called by the first six threads of a block.
__device__ inline void load_face_bases(const int* __restrict__ nbr, int b, int64_t* sb) {
  if (threadIdx.x < 6) {
    const int idx[6] = {nbr_index(-1, 0, 0), nbr_index(1, 0, 0), nbr_index(0, -1, 0),
                        nbr_index(0, 1, 0),  nbr_index(0, 0, -1), nbr_index(0, 0, 1)};
    int nb = nbr[(size_t)b * kNbr + idx[threadIdx.x]];
    sb[threadIdx.x] = nb < 0 ? -1 : (int64_t)nb * kCells;
  }
}

// A domain brick's row of the brick rows built with the solve's domain list:
// its pool index and its -x, +x, -y, +y, -z, +z face neighbours (-1 absent),
// 8 ints. One load round gives a block its brick and face bases (threads 0..5
// stage them, in load_face_bases' order), where the list and the neighbour
// table take two.
__device__ inline int load_drow(const int* __restrict__ drow, int64_t* sb) {
  const int* row = drow + 8 * (size_t)blockIdx.x;
  if (threadIdx.x < 6) {
    const int nb = row[1 + threadIdx.x];
    sb[threadIdx.x] = nb < 0 ? -1 : (int64_t)nb * kCells;
  }
  return row[0];
}

// Index of the face-f neighbour of cell c (slot o of its brick), -1 if its brick is absent.
__device__ inline int64_t nb0(const int64_t* sb, int64_t c, int o, int f) {
  int x = o & 7, y = (o >> 3) & 7, z = o >> 6;
  switch (f) {
    case 0: return x > 0 ? c - 1 : (sb[0] < 0 ? -1 : sb[0] + o + 7);
    case 1: return x < 7 ? c + 1 : (sb[1] < 0 ? -1 : sb[1] + o - 7);
    case 2: return y > 0 ? c - 8 : (sb[2] < 0 ? -1 : sb[2] + o + 56);
    case 3: return y < 7 ? c + 8 : (sb[3] < 0 ? -1 : sb[3] + o - 56);
    case 4: return z > 0 ? c - 64 : (sb[4] < 0 ? -1 : sb[4] + o + 448);
    default: return z < 7 ? c + 64 : (sb[5] < 0 ? -1 : sb[5] + o - 448);
  }
}

// Level-0 brick kernels: one block of kBT threads per brick, kCPT cells per
// thread (slots threadIdx.x + kBT*k), so every thread keeps several
// independent load chains in flight.
constexpr int kBT = 128;
constexpr int kCPT = kCells / kBT;

// Shared-memory staging of one brick with its six face halos: a 10^3 array,
// interior (x,y,z) at (x+1) + 10(y+1) + 100(z+1); edge and corner entries are
// not used by 7-point stencils. val(global index) produces the staged value;
// cells of an absent neighbour brick stage `zero`. All loads are independent,
// so a block has its whole brick in flight at once.
constexpr int kS1 = 1000;
__device__ inline int s1(int x, int y, int z) { return (x + 1) + 10 * (y + 1) + 100 * (z + 1); }
__device__ inline int s1_of(int o) { return s1(o & 7, (o >> 3) & 7, o >> 6); }
__device__ inline int s1_off(int f) {
  const int mag = (f >> 1) == 0 ? 1 : ((f >> 1) == 1 ? 10 : 100);
  return (f & 1) ? mag : -mag;
}

// The face halos: 384 slots, three per thread. Thread t takes position
// (u, v) = (t & 7, (t >> 3) & 7) on the three faces of sign t >> 6 (0: -x,
// -y, -z; 1: +x, +y, +z), one per axis a; the element is cell off of face
// neighbour f's brick (the row of that brick next to this one) and lands in
// staging slot `slot`.
static_assert(kBT == 128, "the halo map gives each of 128 threads three slots");
struct HaloSlot {
  int slot;  // staging slot
  int f;     // face: 2 * axis + sign (the index into the face bases)
  int off;   // cell within the neighbour brick
};
__device__ inline HaloSlot halo_slot(int a) {
  const int t = threadIdx.x & 63, sg = threadIdx.x >> 6, u = t & 7, v = t >> 3;
  const int e = sg ? 8 : -1, w = sg ? 0 : 7;
  HaloSlot h;
  h.f = 2 * a + sg;
  if (a == 0) {
    h.slot = s1(e, u, v);
    h.off = w + 8 * u + 64 * v;
  } else if (a == 1) {
    h.slot = s1(u, e, v);
    h.off = u + 8 * w + 64 * v;
  } else {
    h.slot = s1(u, v, e);
    h.off = u + 8 * v + 64 * w;
  }
  return h;
}

// The same staging of a plain array: the brick's own 512 cells with 16-byte
// vector loads (thread t takes cells 4t..4t+3, half a row), the face halos
// with scalar loads; the values land in s converted to its element type S.
template <class V>
__device__ inline void load4(const double* p, V* v) {
  const double2 a = *reinterpret_cast<const double2*>(p);
  const double2 c = *reinterpret_cast<const double2*>(p + 2);
  v[0] = (V)a.x; v[1] = (V)a.y; v[2] = (V)c.x; v[3] = (V)c.y;
}
template <class V>
__device__ inline void load4(const float* p, V* v) {
  const float4 a = *reinterpret_cast<const float4*>(p);
  v[0] = (V)a.x; v[1] = (V)a.y; v[2] = (V)a.z; v[3] = (V)a.w;
}

// Stencil passes over a staged brick give thread t the z-run of four cells
// (t & 63) + 256 (t >> 6) + 64 k, k = 0..3, of one (x, y) column: the loads
// and stores of each k stay coalesced, and a cell's z neighbours inside the
// run are the thread's own staged values (v[k -+ 1]) rather than shared-memory
// reads; zrun_nbr gives the face-f neighbour of run cell k at staging slot si.
static_assert(kCPT == 4, "z-runs of four cells");
__device__ inline int zrun_base() { return (threadIdx.x & 63) + 256 * (threadIdx.x >> 6); }
template <class S>
__device__ inline S zrun_nbr(const S* s, const S* v, int si, int k, int f) {
  if (f == 4) return k > 0 ? v[k - 1] : s[si - 100];
  if (f == 5) return k < kCPT - 1 ? v[k + 1] : s[si + 100];
  return s[si + s1_off(f)];
}

// The face halos of a brick staging: s[slot] = val(global index), 0 where the
// neighbour brick is absent; all three loads are issued before any store.
template <class S, class F>
__device__ inline void stage_h1_halo(S* s, const int64_t* sb, F val) {
  S hv[3];
  int hs[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const HaloSlot h = halo_slot(a);
    hs[a] = h.slot;
    hv[a] = sb[h.f] < 0 ? (S)0 : (S)val(sb[h.f] + h.off);
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) s[hs[a]] = hv[a];
}

template <class S, class T>
__device__ inline void stage_arr(S* s, const T* __restrict__ a, int b, const int64_t* sb) {
  static_assert(kBT * 4 == kCells, "one 4-cell vector per thread");
  const int o = 4 * threadIdx.x;
  S v[4];
  load4(a + (int64_t)b * kCells + o, v);
  stage_h1_halo(s, sb, [&](int64_t i) { return a[i]; });
  const int si = s1_of(o);
#pragma unroll
  for (int q = 0; q < 4; ++q) s[si + q] = v[q];
}

// Kernels of an iterative solve that the host enqueues ahead of its
// convergence check do nothing once the solve is done (done == nullptr: run).
__device__ inline bool solve_done(const int32_t* done) { return done != nullptr && *done != 0; }

// Sum over an NT-thread block of two values into partial[blockIdx.x] and
// partial[gridDim.x + blockIdx.x] (fixed order).
template <int NT>
__device__ inline void block_sum(double a, double b, double* partial) {
  __shared__ double ra[NT / 32], rb[NT / 32];
  for (int s = 16; s > 0; s >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, s);
    b += __shfl_down_sync(0xffffffffu, b, s);
  }
  if ((threadIdx.x & 31) == 0) {
    ra[threadIdx.x >> 5] = a;
    rb[threadIdx.x >> 5] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0, tb = 0;
    for (int i = 0; i < NT / 32; ++i) {
      ta += ra[i];
      tb += rb[i];
    }
    partial[blockIdx.x] = ta;
    partial[gridDim.x + blockIdx.x] = tb;
  }
}

inline int grid_for(int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  return (int)(g < 1 ? 1 : g);
}

// ------------------------------------------------------------- launchers
// Implemented in the .cu files; all enqueue on ctx->stream.
int check(cudaError_t e);
bool learned_solver(const Ctx* c);
int learned_begin(Ctx* c);
int learned_precondition(Ctx* c, int first);
int topology_rebuild(Ctx* c, bool first_init_order);
int topo_initialize(Ctx* c);
int topo_layer_initial(Ctx* c);
int topo_create_fluid(Ctx* c);
int topo_update_layer(Ctx* c);
int topo_delete(Ctx* c);
int topo_dt(Ctx* c);
int topo_finish(Ctx* c);
int rebuild_index(Ctx* c);
int read_scalars(Ctx* c);
int forces(Ctx* c, int ib);
int rk2tvd(Ctx* c);
int project(Ctx* c, int ib);
int project_field(Ctx* c, double* const* U, const double* const* D);
int extrapolate_field(Ctx* c, double* const* F);
int forces_add(Ctx* c, const double* const* U);
int rk_all_stage_update(Ctx* c, int stage, const double* const* U);
int acc_zero(Ctx* c);
int topology_stage(Ctx* c);
int setup_system(Ctx* c);
int extrapolate(Ctx* c);
int move_particles(Ctx* c);
// The move's two halves: binning the particles by brick and cell on stream st
// (into the second particle buffers, which then become the current ones), and
// the RK4 move of the binned particles on the context's stream.
int bin_particles(Ctx* c, cudaStream_t st);
int move_binned(Ctx* c);
// Starts the pending binning on the side stream (once per step, at the first
// projection's CG loop, where the device is latency-bound).
int launch_side_binning(Ctx* c);
int alloc_solver(Ctx* c);
void free_solver(Ctx* c);
int mg_setup(Ctx* c);
// update = 1: the V-cycle's first kernel also applies the previous CG
// iteration's x += alpha p, r -= alpha q and its convergence test. part: 1 =
// that first kernel (and the test), 2 = the rest of the V-cycle, 3 = all.
void mg_vcycle(Ctx* c, int update, int part);
void cg_finish_update(Ctx* c);
int mg_configure(Ctx* c);

}  // namespace mac
