// Advection stage on the brick grid: gravity + first-order upwind convection
// fused with the SSP-RK2 stage updates, air-layer velocity extrapolation and
// the RK4 particle move through the staggered trilinear field.
//
// The library is compiled with -fmad=false and every expression keeps the
// reference's operation order, so these kernels reproduce the reference's
// FP64 results bit for bit from the same input state.
#include <utility>

#include "mac_internal.cuh"

namespace mac {

// Index of the cell at local coordinates (x,y,z) of the brick whose
// neighbour row is `sn` (coordinates may leave the brick by up to one brick);
// -1 when that brick is not live.
__device__ inline int64_t cidx(const int* sn, int x, int y, int z) {
  int dx = x < 0 ? -1 : (x >= 8 ? 1 : 0);
  int dy = y < 0 ? -1 : (y >= 8 ? 1 : 0);
  int dz = z < 0 ? -1 : (z >= 8 ? 1 : 0);
  int b = sn[nbr_index(dx, dy, dz)];
  if (b < 0) return -1;
  return (int64_t)b * kCells + ((x - 8 * dx) + 8 * (y - 8 * dy) + 64 * (z - 8 * dz));
}

// Speed read: a cell the reference would dereference through a null chunk
// (src/Offset_Base_Neighbour.h:14-33) reads 0 here.
__device__ inline double rdv(const double* __restrict__ U, int64_t i) { return i < 0 ? 0.0 : U[i]; }

// The brick of a force kernel and its halo in shared memory, slot s1(x, y, z)
// for coordinates -1..8: the three speed components (0 where the brick is not
// live, as rdv reads), the layer (kMissing there) and the material. The
// stencils below read the brick, its face halos and the edge cells
// c - e_i + e_j; corner slots are never read and stay unset.
struct Stage {
  double u[3][kS1];
  int8_t lay[kS1];
  uint8_t type[kS1];
};

__device__ inline void stage_forces(Stage& S, const double* const* U, const int* sn, const int8_t* __restrict__ lay,
                                    const uint8_t* __restrict__ type) {
  for (int t = threadIdx.x; t < kS1; t += blockDim.x) {
    const int x = t % 10 - 1, y = (t / 10) % 10 - 1, z = t / 100 - 1;
    if ((x < 0 || x > 7) + (y < 0 || y > 7) + (z < 0 || z > 7) > 2) continue;
    const int64_t i = cidx(sn, x, y, z);
    S.u[0][t] = rdv(U[0], i);
    S.u[1][t] = rdv(U[1], i);
    S.u[2][t] = rdv(U[2], i);
    S.lay[t] = i < 0 ? kMissing : lay[i];
    S.type[t] = i < 0 ? (uint8_t)0 : type[i];
  }
}

__device__ inline double su(const Stage& S, int j, int x, int y, int z) { return S.u[j][s1(x, y, z)]; }

// The cell at (x, y, z) exists and is fluid (false where its brick is not live).
__device__ inline bool fluid_at(const Stage& S, int x, int y, int z) {
  const int t = s1(x, y, z);
  return S.lay[t] != kMissing && is_fluid(S.type[t]);
}

// Get_Speed_At_Bound (src/Policy_Speed_Interpolation_Linear_Symmetric.h:120-127,
// identical in src/Policy_Speed_Interpolation_Linear.h:107-114).
__device__ inline double speed_at_bound(const Stage& S, int x, int y, int z, int i, int j) {
  if (i == j) return su(S, j, x, y, z);
  int cj[3] = {x, y, z}, ci[3] = {x, y, z}, cij[3] = {x, y, z};
  cj[j] += 1;
  ci[i] -= 1;
  cij[i] -= 1;
  cij[j] += 1;
  double a = su(S, j, x, y, z);
  double b = su(S, j, cj[0], cj[1], cj[2]);
  double d = su(S, j, ci[0], ci[1], ci[2]);
  double e = su(S, j, cij[0], cij[1], cij[2]);
  return 0.25 * (((a + b) + d) + e);
}

// Policy_Upwind_1_Order::Get_Convection_Speed(neigh, i) (src/Policy_Upwind_1_Order.h:18-38,58-66).
__device__ inline double convection(const Stage& S, int x, int y, int z, int i, const Params& P) {
  double ret = 0;
  double U1 = su(S, i, x, y, z);
  for (int j = 0; j < 3; ++j) {
    double Ub = speed_at_bound(S, x, y, z, i, j);
    int m[3] = {x, y, z};
    if (Ub > 0) {
      m[j] -= 1;
      double U2 = su(S, i, m[0], m[1], m[2]);
      Ub *= (U1 - U2) * P.ih[j];
    } else {
      m[j] += 1;
      double U2 = su(S, i, m[0], m[1], m[2]);
      Ub *= (U2 - U1) * P.ih[j];
    }
    ret -= Ub;
  }
  return ret;
}

// Policy_Viscosity_Apply_If::Get_Viscosity_Apply_If (src/Policy_Viscosity_Apply_If.h:15-42):
// a fluid cell, or a cell with a layer one of whose -e_j neighbours (any axis)
// exists and is fluid. One answer for the three faces of the cell.
__device__ inline bool viscosity_applies(const Stage& S, bool fluid, int x, int y, int z) {
  if (fluid) return true;
  if (S.lay[s1(x, y, z)] == kEmpty) return false;
  for (int j = 0; j < 3; ++j)
    if (fluid_at(S, x - (j == 0), y - (j == 1), z - (j == 2))) return true;
  return false;
}

// Policy_Laplacian_Speed::Get_Laplacian_Speed(neigh, i) (src/Policy_Laplacian_Speed.h:22-36):
// per axis j, -2 u(c)/h_j^2 + u(c+e_j)/h_j^2 + u(c-e_j)/h_j^2 with h_j^-2 = pow(1/h_j, 2),
// accumulated in that order.
__device__ inline double laplacian(const Stage& S, int i, int x, int y, int z, const Params& P) {
  double t = 0;
  const double uc = su(S, i, x, y, z);
  for (int j = 0; j < 3; ++j) {
    t -= 2 * uc * P.lih2[j];
    t += su(S, i, x + (j == 0), y + (j == 1), z + (j == 2)) * P.lih2[j];
    t += su(S, i, x - (j == 0), y - (j == 1), z - (j == 2)) * P.lih2[j];
  }
  return t;
}

// Acceleration of face i of cell (x,y,z): forced zero, then Policy_Gravity and
// Policy_Upwind_1_Order applied through the non-forced Set (const faces keep 0).
// Gravity applies if the cell is fluid, or has a layer and its -e_g neighbour
// is fluid (src/Policy_Gravity.h:14-34); convection uses the same rule on axis
// i (src/Policy_Convection_Apply_If.h:41-61). With a viscosity, Algorithms_Viscosity
// (src/Algorithms_Viscosity.h:24-30) then adds viscosity * Laplacian.
// base: the acceleration the contributions add to (0 after the forced zero;
// pipeline B's stage forces add to what a re-created cell holds).
__device__ inline double face_accel(const Stage& S, uint8_t fl, int x, int y, int z, int i, const Params& P,
                                    double base = 0.0) {
  if (fl & (1u << i)) return base;
  const int sc = s1(x, y, z);
  bool fluid = is_fluid(S.type[sc]);
  // convection and gravity on axis i: the cell is fluid, or it has a layer
  // and its -e_i neighbour exists and is fluid
  bool apply = fluid || (S.lay[sc] != kEmpty && fluid_at(S, x - (i == 0), y - (i == 1), z - (i == 2)));
  double a = base;
  if (i == P.gaxis && apply) a = a + P.g;
  if (apply) a = a + convection(S, x, y, z, i, P);
  if (P.nu != 0.0 && viscosity_applies(S, fluid, x, y, z)) a = a + laplacian(S, i, x, y, z, P) * P.nu;
  return a;
}

// mode 0: acc = forces(u[ib]); mode 1: RK stage 1 (src/Algorithms_RungeKutta_RK2_TVD.h:31-43):
// u1 = u0 + a(u0)*dt, forced; mode 2: stage 2 (:45-58 after the first projection):
// acc = a(u1) and u0 = 0.5*u0 + 0.5*u1 + 0.5*acc*dt through the non-forced Set.
// The speed field read by the stencils is staged per brick; the kernels write
// other arrays only, so no block reads what another writes.
template <int MODE>
__global__ void __launch_bounds__(256) k_forces(const int* __restrict__ blist, int nlive, const int* __restrict__ nbr,
                                                const int8_t* __restrict__ lay, const uint8_t* __restrict__ type,
                                                const uint8_t* __restrict__ flags, double* f64, size_t cap,
                                                int ib, Params P, const Scalars* __restrict__ ds) {
  __shared__ int sn[kNbr];
  __shared__ Stage S;
  const double dt = ds->dt;
  const double* U[3];
  for (int i = 0; i < 3; ++i) U[i] = f64 + (size_t)((MODE == 2 ? 1 : (MODE == 1 ? 0 : ib)) * 3 + i) * cap;
  for (int bi = blockIdx.x; bi < nlive; bi += gridDim.x) {
    int b = blist[bi];
    if (threadIdx.x < kNbr) sn[threadIdx.x] = nbr[(size_t)b * kNbr + threadIdx.x];
    __syncthreads();
    stage_forces(S, U, sn, lay, type);
    __syncthreads();
    for (int o = threadIdx.x; o < kCells; o += blockDim.x) {
      int64_t c = (int64_t)b * kCells + o;
      int x = o & 7, y = (o >> 3) & 7, z = o >> 6;
      if (S.lay[s1(x, y, z)] == kMissing) continue;
      uint8_t fl = flags[c];
      double a[3];
      for (int i = 0; i < 3; ++i) a[i] = face_accel(S, fl, x, y, z, i, P);
      if (MODE == 0) {
        for (int i = 0; i < 3; ++i) f64[(size_t)(AX + i) * cap + c] = a[i];
      } else if (MODE == 1) {
        for (int i = 0; i < 3; ++i)
          f64[(size_t)(U1X + i) * cap + c] = S.u[i][s1(x, y, z)] + a[i] * dt;
      } else {
        for (int i = 0; i < 3; ++i) {
          f64[(size_t)(AX + i) * cap + c] = a[i];
          if (!(fl & (1u << i))) {
            double u0 = f64[(size_t)(U0X + i) * cap + c], u1 = S.u[i][s1(x, y, z)];
            f64[(size_t)(U0X + i) * cap + c] = 0.5 * u0 + 0.5 * u1 + 0.5 * a[i] * dt;
          }
        }
      }
    }
    __syncthreads();
  }
}

// Pipeline B's Algorithms<Gravity, Convection, Viscosity> of a stage: acc +=
// the forces of speed field U, through the non-forced Set, for every existing
// cell (src/Algorithms_Gravity.h:15-28, src/Algorithms_Convection.h:18-37,
// src/Algorithms_Viscosity.h:24-30).
__global__ void __launch_bounds__(256) k_forces_add(const int* __restrict__ blist, int nlive,
                                                    const int* __restrict__ nbr, const int8_t* __restrict__ lay,
                                                    const uint8_t* __restrict__ type, const uint8_t* __restrict__ flags,
                                                    const double* __restrict__ ux, const double* __restrict__ uy,
                                                    const double* __restrict__ uz, double* ax, double* ay, double* az,
                                                    Params P) {
  __shared__ int sn[kNbr];
  __shared__ Stage S;
  const double* U[3] = {ux, uy, uz};
  double* A[3] = {ax, ay, az};
  for (int bi = blockIdx.x; bi < nlive; bi += gridDim.x) {
    int b = blist[bi];
    if (threadIdx.x < kNbr) sn[threadIdx.x] = nbr[(size_t)b * kNbr + threadIdx.x];
    __syncthreads();
    stage_forces(S, U, sn, lay, type);
    __syncthreads();
    for (int o = threadIdx.x; o < kCells; o += blockDim.x) {
      int64_t c = (int64_t)b * kCells + o;
      int x = o & 7, y = (o >> 3) & 7, z = o >> 6;
      if (S.lay[s1(x, y, z)] == kMissing) continue;
      uint8_t fl = flags[c];
      double a[3];
      for (int i = 0; i < 3; ++i) a[i] = face_accel(S, fl, x, y, z, i, P, A[i][c]);
      for (int i = 0; i < 3; ++i) A[i][c] = a[i];
    }
    __syncthreads();
  }
}

int forces_add(Ctx* c, const double* const* U) {
  if (c->nlive_host == 0) return MAC_OK;
  size_t cap = (size_t)c->cap_bricks * kCells;
  prof_begin(c, PH_FORCES);
  k_forces_add<<<c->nlive_host, 256, 0, c->stream>>>(c->blist, c->nlive_host, c->nbr, c->lay, c->type, c->flags,
                                                     U[0], U[1], U[2], c->f64 + AX * cap, c->f64 + AY * cap,
                                                     c->f64 + AZ * cap, c->dp); MAC_COUNT(c);
  prof_end(c, PH_FORCES);
  return check(cudaGetLastError());
}

int forces(Ctx* c, int ib) {
  if (c->nlive_host == 0) return MAC_OK;
  size_t cap = (size_t)c->cap_bricks * kCells;
  k_forces<0><<<c->nlive_host, 256, 0, c->stream>>>(c->blist, c->nlive_host, c->nbr, c->lay, c->type, c->flags,
                                                    c->f64, cap, ib, c->dp, c->ds); MAC_COUNT(c);
  return check(cudaGetLastError());
}

int rk_stage(Ctx* c, int stage) {
  if (c->nlive_host == 0) return MAC_OK;
  size_t cap = (size_t)c->cap_bricks * kCells;
  prof_begin(c, PH_FORCES);
  if (stage == 1) {
    k_forces<1><<<c->nlive_host, 256, 0, c->stream>>>(c->blist, c->nlive_host, c->nbr, c->lay, c->type, c->flags,
                                                      c->f64, cap, 0, c->dp, c->ds); MAC_COUNT(c);
  } else {
    k_forces<2><<<c->nlive_host, 256, 0, c->stream>>>(c->blist, c->nlive_host, c->nbr, c->lay, c->type, c->flags,
                                                      c->f64, cap, 1, c->dp, c->ds); MAC_COUNT(c);
  }
  prof_end(c, PH_FORCES);
  return check(cudaGetLastError());
}

// ------------------------------------------------------------ extrapolation
// Algorithms_Extrapolate::Do (src/Algorithms_Extrapolate.h:25-233), one launch
// per level L. A face u_i(c) (between A = c - e_i and c) is written at level L
// when A has layer L and c a layer >= L (the "+1 direction" branch of a layer-L
// cell, :56-115), when c has layer L and A a layer >= L (the "-1 direction"
// branch, :117-176) or when c has layer L and A is missing or empty (:177-220).
// The first two compute the same ordered sum, so every face has one value; the
// faces read are those touching a layer < L, final before level L starts, so a
// level is race-free. n == 0 gives 0/0 like the reference.
__device__ inline int8_t lay_i(const int8_t* __restrict__ lay, int64_t i) { return i < 0 ? kMissing : lay[i]; }

__device__ inline uint32_t layer_bit(int l) { return 1u << (l < 31 ? l : 31); }

// The layers present in each live brick (bit l for layer l), so that a level's
// launch skips the bricks it cannot write.
__global__ void __launch_bounds__(256) k_layer_mask(const int* __restrict__ blist, const int8_t* __restrict__ lay,
                                                    uint32_t* __restrict__ lmask) {
  __shared__ uint32_t sw[8];
  const int b = blist[blockIdx.x];
  uint32_t m = 0;
  for (int o = threadIdx.x; o < kCells; o += blockDim.x) {
    const int8_t l = lay[(int64_t)b * kCells + o];
    if (l >= 0) m |= layer_bit(l);
  }
  m = __reduce_or_sync(0xffffffffu, m);
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < 8; ++w) m |= sw[w];
    lmask[b] = m;
  }
}

// A face of a cell in brick b is written at level L only when its cell or the
// cell behind it (-e_i) has layer L, so only when b or one of its -x, -y, -z
// face neighbours holds a layer-L cell; other bricks are skipped whole.
__global__ void __launch_bounds__(256) k_extrapolate(const int* __restrict__ blist, int nlive, const int* __restrict__ nbr,
                                                     const int8_t* __restrict__ lay, const uint8_t* __restrict__ flags,
                                                     const uint32_t* __restrict__ lmask, double* fx, double* fy,
                                                     double* fz, int L) {
  double* const F[3] = {fx, fy, fz};
  __shared__ int sn[kNbr];
  for (int bi = blockIdx.x; bi < nlive; bi += gridDim.x) {
    int b = blist[bi];
    if (threadIdx.x < kNbr) sn[threadIdx.x] = nbr[(size_t)b * kNbr + threadIdx.x];
    __syncthreads();
    uint32_t near = lmask[b];
    for (int i = 0; i < 3; ++i) {
      const int nb = sn[nbr_index(i == 0 ? -1 : 0, i == 1 ? -1 : 0, i == 2 ? -1 : 0)];
      if (nb >= 0) near |= lmask[nb];
    }
    const bool skip = !(near & layer_bit(L));
    for (int o = skip ? kCells : threadIdx.x; o < kCells; o += blockDim.x) {
      int64_t c = (int64_t)b * kCells + o;
      int8_t lB = lay[c];
      if (lB < 0) continue;  // c must exist with a layer
      int x = o & 7, y = (o >> 3) & 7, z = o >> 6;
      uint8_t fl = flags[c];
      for (int i = 0; i < 3; ++i) {
        if (fl & (1u << i)) continue;  // non-forced Set on a const face does nothing
        int a[3] = {x, y, z};
        a[i] -= 1;
        int8_t lA = lay_i(lay, cidx(sn, a[0], a[1], a[2]));
        bool vA = lA >= 0;
        bool write = (vA && lA == L && lB >= L) || (lB == L && (!vA || lA >= L));
        if (!write) continue;
        const double* Ui = F[i];
        int n = 0;
        double val = 0;
        for (int j = 0; j < 3; ++j) {
          for (int s = -1; s <= 1; s += 2) {
            if (j == i) {
              if (s == -1) {
                if (!vA) continue;
                int m[3] = {x, y, z};
                m[i] -= 2;
                int8_t l = lay_i(lay, cidx(sn, m[0], m[1], m[2]));
                if (l >= 0 && l < L) {
                  ++n;
                  val += rdv(Ui, cidx(sn, a[0], a[1], a[2]));
                }
              } else {
                int m[3] = {x, y, z};
                m[i] += 1;
                int64_t mi = cidx(sn, m[0], m[1], m[2]);
                int8_t l = lay_i(lay, mi);
                if (l >= 0 && l < L) {
                  ++n;
                  val += rdv(Ui, mi);
                }
              }
            } else {
              int m4[3] = {x, y, z};
              m4[j] += s;
              int m3[3] = {m4[0], m4[1], m4[2]};
              m3[i] -= 1;
              int64_t i4 = cidx(sn, m4[0], m4[1], m4[2]);
              int8_t l4 = lay_i(lay, i4);
              int8_t l3 = lay_i(lay, cidx(sn, m3[0], m3[1], m3[2]));
              if (l3 >= 0 && l4 >= 0 && (l3 < L || l4 < L)) {
                ++n;
                val += rdv(Ui, i4);
              }
            }
          }
        }
        F[i][c] = val / n;
      }
    }
    __syncthreads();
  }
}

// Algorithms_Extrapolate on the vector field F (speed buffer 0 in pipeline A;
// the stage speed and, through Algorithms_Accel_To_Speed, the acceleration in
// pipeline B).
int extrapolate_field(Ctx* c, double* const* F) {
  if (c->nlive_host == 0) return MAC_OK;
  prof_begin(c, PH_EXTRAPOLATE);
  k_layer_mask<<<c->nlive_host, 256, 0, c->stream>>>(c->blist, c->lay, c->lmask); MAC_COUNT(c);
  for (int L = 1; L <= c->dp.layer_max + 1; ++L) {
    k_extrapolate<<<c->nlive_host, 256, 0, c->stream>>>(c->blist, c->nlive_host, c->nbr, c->lay, c->flags, c->lmask,
                                                        F[0], F[1], F[2], L); MAC_COUNT(c);
  }
  prof_end(c, PH_EXTRAPOLATE);
  return check(cudaGetLastError());
}

int extrapolate(Ctx* c) {
  size_t cap = (size_t)c->cap_bricks * kCells;
  double* F[3] = {c->f64 + U0X * cap, c->f64 + U0Y * cap, c->f64 + U0Z * cap};
  return extrapolate_field(c, F);
}

// ---------------------------------------------------------------- particles
// Staggered trilinear interpolation Get_Speed (src/Policy_Speed_Interpolation_Linear_Symmetric.h:79-119
// when sym, src/Policy_Speed_Interpolation_Linear.h:64-106 otherwise): the 2x2x2
// stencil of component k around key0 = lround(pos/h), weights (1-d, d) off-axis
// and (1/2-d, 1/2+d) on axis k (the non-symmetric variant shifts d_k by 1/2),
// combined x-outermost as the reference's recursion does.
struct PBase {
  int key[3];  // base brick key
  int b;       // its pool index (-1 if missing)
};

__device__ inline int64_t pcell(const PBase& pb, const int* __restrict__ nbr, const unsigned long long* __restrict__ hk,
                                const int* __restrict__ hv, int64_t hcap, int kx, int ky, int kz) {
  int bx = fdiv8(kx), by = fdiv8(ky), bz = fdiv8(kz);
  int dx = bx - pb.key[0], dy = by - pb.key[1], dz = bz - pb.key[2];
  int b;
  if (pb.b >= 0 && dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1 && dz >= -1 && dz <= 1)
    b = nbr[(size_t)pb.b * kNbr + nbr_index(dx, dy, dz)];
  else
    b = hash_find(hk, hv, hcap, pack_key(bx, by, bz));
  if (b < 0) return -1;
  return (int64_t)b * kCells + (kx & 7) + 8 * (ky & 7) + 64 * (kz & 7);
}

// Field read through the brick table (any cell; used for particles whose
// stencil leaves the staged region and for unbinned particles).
struct GlobalField {
  PBase pb;
  const int* nbr;
  const unsigned long long* hk;
  const int* hv;
  int64_t hcap;
  const int8_t* lay;
  const double* const* U;
  __device__ double u(int k, int kx, int ky, int kz, int* bad) const {
    int64_t ci = pcell(pb, nbr, hk, hv, hcap, kx, ky, kz);
    if (ci < 0 || lay[ci] == kMissing) *bad = 1;
    return ci < 0 ? 0.0 : U[k][ci];
  }
};

// Field read from a shared-memory copy of the 12^3 region around a brick
// (its cells with a two-cell halo), falling back to the brick table outside it.
constexpr int kStage = 12;
constexpr int kStageCells = kStage * kStage * kStage;
// Shared-memory layout of the staged field: slot x + kStage y + kStageZ z per
// component, components kStageComp apart. A z-stride of kStage^2 = 144
// doubles is a multiple of the 32 four-byte banks, so the 2x2x2 stencil's
// z-pairs of neighbouring particles hit the same banks; one padding double per
// z-plane moves them two banks apart.
constexpr int kStageZ = kStage * kStage + 1;
constexpr int kStageComp = kStageZ * kStage;
__host__ __device__ constexpr int stage_slot(int x, int y, int z) { return x + kStage * y + kStageZ * z; }
struct StagedField {
  const double* s;        // [3][kStageComp]
  int ox, oy, oz;         // cell key of stage slot (0,0,0)
  GlobalField g;
  __device__ double u(int k, int kx, int ky, int kz, int* bad) const {
    unsigned x = (unsigned)(kx - ox), y = (unsigned)(ky - oy), z = (unsigned)(kz - oz);
    if (x < (unsigned)kStage && y < (unsigned)kStage && z < (unsigned)kStage)
      return s[k * kStageComp + stage_slot((int)x, (int)y, (int)z)];
    return g.u(k, kx, ky, kz, bad);
  }
  // The 2x2x2 stencil of component k at corner key (index n = 4X + 2Y + Z);
  // one bounds test for the whole stencil.
  __device__ void u8(int k, const int* key, double* out, int* bad) const {
    unsigned x = (unsigned)(key[0] - ox), y = (unsigned)(key[1] - oy), z = (unsigned)(key[2] - oz);
    if (x + 1 < (unsigned)kStage && y + 1 < (unsigned)kStage && z + 1 < (unsigned)kStage) {
      const double* p = s + k * kStageComp + stage_slot((int)x, (int)y, (int)z);
      out[0] = p[0];
      out[1] = p[kStageZ];
      out[2] = p[kStage];
      out[3] = p[kStage + kStageZ];
      out[4] = p[1];
      out[5] = p[1 + kStageZ];
      out[6] = p[1 + kStage];
      out[7] = p[1 + kStage + kStageZ];
      return;
    }
#pragma unroll
    for (int n = 0; n < 8; ++n) out[n] = g.u(k, key[0] + (n >> 2), key[1] + ((n >> 1) & 1), key[2] + (n & 1), bad);
  }
};

template <class F>
__device__ inline void stencil8(const F& field, int k, const int* key, double* u, int* bad) {
#pragma unroll
  for (int n = 0; n < 8; ++n) u[n] = field.u(k, key[0] + (n >> 2), key[1] + ((n >> 1) & 1), key[2] + (n & 1), bad);
}
__device__ inline void stencil8(const StagedField& field, int k, const int* key, double* u, int* bad) {
  field.u8(k, key, u, bad);
}

template <class F>
__device__ inline void get_speed(const double* pos, double* out, const F& field, const Params& P, int sym, int* bad) {
  double pd[3];
  int k0[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    pd[i] = pos[i] * P.ih[i];
    k0[i] = (int)lround(pd[i]);
    pd[i] -= k0[i];
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (!sym) pd[k] += 0.5;
    int key[3];
    double d[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      if (j != k && pd[j] < 0) {
        key[j] = k0[j] - 1;
        d[j] = 1 + pd[j];
      } else {
        key[j] = k0[j];
        d[j] = pd[j];
      }
    }
    double w0[3], w1[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      if (sym && i == k) {
        w0[i] = 0.5 - d[i];
        w1[i] = 0.5 + d[i];
      } else {
        w0[i] = 1 - d[i];
        w1[i] = d[i];
      }
    }
    double u[8];
    stencil8(field, k, key, u, bad);
    // u[(X<<2)|(Y<<1)|Z]
    double l00 = w0[2] * u[0] + w1[2] * u[1];
    double l01 = w0[2] * u[2] + w1[2] * u[3];
    double l10 = w0[2] * u[4] + w1[2] * u[5];
    double l11 = w0[2] * u[6] + w1[2] * u[7];
    double m0 = w0[1] * l00 + w1[1] * l01;
    double m1 = w0[1] * l10 + w1[1] * l11;
    out[k] = w0[0] * m0 + w1[0] * m1;
    if (!sym) pd[k] -= 0.5;
  }
}

// Policy_Advance_Ode_RungeKutta::AdvanceSolveODE (src/Policy_Advance_ODE_RungeKutta.h:15-27):
// classic RK4 in this accumulation order.
template <class F>
__device__ inline void rk4(double* pos, const F& field, const Params& P, double dt, int* bad) {
  double res[3], k[3], a[3], v[3];
  for (int i = 0; i < 3; ++i) res[i] = pos[i];
  get_speed(pos, v, field, P, P.interp_sym, bad);
  for (int i = 0; i < 3; ++i) {
    k[i] = dt * v[i];
    res[i] += (1. / 6.) * k[i];
  }
  for (int i = 0; i < 3; ++i) a[i] = pos[i] + k[i] * 0.5;
  get_speed(a, v, field, P, P.interp_sym, bad);
  for (int i = 0; i < 3; ++i) {
    k[i] = dt * v[i];
    res[i] += (1. / 3.) * k[i];
  }
  for (int i = 0; i < 3; ++i) a[i] = pos[i] + k[i] * 0.5;
  get_speed(a, v, field, P, P.interp_sym, bad);
  for (int i = 0; i < 3; ++i) {
    k[i] = dt * v[i];
    res[i] += (1. / 3.) * k[i];
  }
  for (int i = 0; i < 3; ++i) a[i] = pos[i] + k[i];
  get_speed(a, v, field, P, P.interp_sym, bad);
  for (int i = 0; i < 3; ++i) {
    k[i] = dt * v[i];
    res[i] += (1. / 6.) * k[i];
  }
  for (int i = 0; i < 3; ++i) pos[i] = res[i];
}

// Particles are binned by the brick of their cell each step, and inside a
// brick's bin by cell (counting sort over 512 * brick + cell; the order inside
// a cell is unspecified). Every particle moves independently, so the order
// changes no result; cell order makes the lanes of a warp read the same
// staged stencil values, which shared memory serves as broadcasts.
__global__ void k_bin_count(const double* __restrict__ px, const double* __restrict__ py,
                            const double* __restrict__ pz, int64_t np, Params P,
                            const unsigned long long* __restrict__ hk, const int* __restrict__ hv, int64_t hcap,
                            int* pbrick, int* ccount, int stray) {
  // Whole warps iterate together so the lanes that share a cell can add their
  // count with one atomic (the array stays mostly sorted from the last step).
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t q0 = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); q0 < np; q0 += stride) {
    int64_t q = q0 + (threadIdx.x & 31);
    int key = -2;
    if (q < np) {
      const int kx = (int)lround(px[q] * P.ih[0]);
      const int ky = (int)lround(py[q] * P.ih[1]);
      const int kz = (int)lround(pz[q] * P.ih[2]);
      int b = hash_find(hk, hv, hcap, pack_key(fdiv8(kx), fdiv8(ky), fdiv8(kz)));
      key = b < 0 ? stray * kCells : b * kCells + (kx & 7) + 8 * (ky & 7) + 64 * (kz & 7);
      pbrick[q] = key;
    }
    unsigned peers = __match_any_sync(0xffffffffu, key);
    int leader = __ffs(peers) - 1;
    if (key >= 0 && (int)(threadIdx.x & 31) == leader) atomicAdd(&ccount[key], __popc(peers));
  }
}

// Per brick of the live list (and the no-brick slot in the last block):
// exclusive scan of its 512 cell counts in place, and the brick total.
__global__ void __launch_bounds__(512) k_cell_scan(const int* __restrict__ blist, int nlive, int stray, int* ccount,
                                                   int* bcount) {
  __shared__ int ws[16];
  const int b = blockIdx.x < nlive ? blist[blockIdx.x] : stray;
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const int v = ccount[(size_t)b * kCells + t];
  int x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) ws[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int w = lane < 16 ? ws[lane] : 0;
#pragma unroll
    for (int d = 1; d < 16; d <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, d);
      if (lane >= d) w += y;
    }
    if (lane < 16) ws[lane] = w;
  }
  __syncthreads();
  const int incl = x + (wid > 0 ? ws[wid - 1] : 0);
  ccount[(size_t)b * kCells + t] = incl - v;
  if (t == kCells - 1) bcount[b] = incl;
}

// Exclusive scan of n counts (one block of 1024 threads).
__global__ void __launch_bounds__(1024) k_bin_scan(const int* __restrict__ cnt, int64_t* __restrict__ off, int n) {
  __shared__ int64_t part[1024];
  int per = (n + 1023) / 1024;
  int lo = threadIdx.x * per, hi = lo + per < n ? lo + per : n;
  int64_t s = 0;
  for (int i = lo; i < hi; ++i) s += cnt[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) {
    int64_t v = threadIdx.x >= d ? part[threadIdx.x - d] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int64_t base = threadIdx.x ? part[threadIdx.x - 1] : 0;
  for (int i = lo; i < hi; ++i) {
    off[i] = base;
    base += cnt[i];
  }
  if (threadIdx.x == 1023) off[n] = part[1023];
}

__global__ void k_bin_scatter(const double* __restrict__ px, const double* __restrict__ py,
                              const double* __restrict__ pz, int64_t np, const int* __restrict__ pbrick,
                              const int64_t* __restrict__ off, int* cursor, double* qx, double* qy, double* qz) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int lane = threadIdx.x & 31;
  for (int64_t q0 = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); q0 < np; q0 += stride) {
    int64_t q = q0 + lane;
    int key = q < np ? pbrick[q] : -2;
    unsigned peers = __match_any_sync(0xffffffffu, key);
    int leader = __ffs(peers) - 1;
    int base = 0;
    if (key >= 0 && lane == leader) base = atomicAdd(&cursor[key], __popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (key >= 0) {
      int64_t pos = off[key / kCells] + base + __popc(peers & ((1u << lane) - 1));
      qx[pos] = px[q];
      qy[pos] = py[q];
      qz[pos] = pz[q];
    }
  }
}

// Algorithms_Move_Particles::Do (src/Algorithms_Move_Particles.h:29-32) for
// the particles binned to one brick: the brick's speed field with a two-cell
// halo (12^3 cells from up to 27 bricks) is staged in shared memory and the
// 96 stencil reads of each particle's RK4 come from there.
__global__ void __launch_bounds__(256) k_move_binned(double* px, double* py, double* pz,
                                                     const int* __restrict__ blist, const int* __restrict__ bkey,
                                                     const int* __restrict__ nbr, const int64_t* __restrict__ off,
                                                     const unsigned long long* __restrict__ hk, const int* __restrict__ hv,
                                                     int64_t hcap, const int8_t* __restrict__ lay,
                                                     const double* __restrict__ ux, const double* __restrict__ uy,
                                                     const double* __restrict__ uz, Params P,
                                                     const Scalars* __restrict__ ds, unsigned long long* bad_count) {
  __shared__ double s[3 * kStageComp];
  __shared__ int sn[kNbr];
  int b = blist[blockIdx.x];
  int64_t p0 = off[b], p1 = off[b + 1];
  if (p0 == p1) return;
  if (threadIdx.x < kNbr) sn[threadIdx.x] = nbr[(size_t)b * kNbr + threadIdx.x];
  __syncthreads();
  const double* U[3] = {ux, uy, uz};
  int ox = bkey[3 * b] * 8 - 2, oy = bkey[3 * b + 1] * 8 - 2, oz = bkey[3 * b + 2] * 8 - 2;
  for (int i = threadIdx.x; i < kStageCells; i += blockDim.x) {
    int x = i % kStage, y = (i / kStage) % kStage, z = i / (kStage * kStage);
    int lx = x - 2, ly = y - 2, lz = z - 2;  // local coordinates in brick b, -2..9
    int dx = lx < 0 ? -1 : (lx >= 8 ? 1 : 0), dy = ly < 0 ? -1 : (ly >= 8 ? 1 : 0), dz = lz < 0 ? -1 : (lz >= 8 ? 1 : 0);
    int nb = sn[nbr_index(dx, dy, dz)];
    const int j = stage_slot(x, y, z);
    if (nb < 0) {
      s[j] = s[kStageComp + j] = s[2 * kStageComp + j] = 0.0;
    } else {
      int64_t gi = (int64_t)nb * kCells + (lx - 8 * dx) + 8 * (ly - 8 * dy) + 64 * (lz - 8 * dz);
      s[j] = U[0][gi];
      s[kStageComp + j] = U[1][gi];
      s[2 * kStageComp + j] = U[2][gi];
    }
  }
  __syncthreads();
  const double dt = ds->dt;
  PBase pb;
  pb.key[0] = bkey[3 * b];
  pb.key[1] = bkey[3 * b + 1];
  pb.key[2] = bkey[3 * b + 2];
  pb.b = b;
  StagedField f{s, ox, oy, oz, GlobalField{pb, nbr, hk, hv, hcap, lay, U}};
  int bad = 0;
  for (int64_t q = p0 + threadIdx.x; q < p1; q += blockDim.x) {
    double pos[3] = {px[q], py[q], pz[q]};
    rk4(pos, f, P, dt, &bad);
    px[q] = pos[0];
    py[q] = pos[1];
    pz[q] = pos[2];
  }
  if (bad) atomicAdd(bad_count, 1ull);
}

// Particles whose cell has no brick (never the case in a valid state; the
// reference would create the cell) move through the brick table.
__global__ void __launch_bounds__(256) k_move_stray(double* px, double* py, double* pz, const int64_t* __restrict__ off,
                                                    int stray, const int* __restrict__ nbr,
                                                    const unsigned long long* __restrict__ hk, const int* __restrict__ hv,
                                                    int64_t hcap, const int8_t* __restrict__ lay,
                                                    const double* __restrict__ ux, const double* __restrict__ uy,
                                                    const double* __restrict__ uz, Params P,
                                                    const Scalars* __restrict__ ds, unsigned long long* bad_count) {
  const double dt = ds->dt;
  const double* U[3] = {ux, uy, uz};
  int bad = 0;
  for (int64_t q = off[stray] + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < off[stray + 1];
       q += (int64_t)gridDim.x * blockDim.x) {
    double pos[3] = {px[q], py[q], pz[q]};
    PBase pb;
    for (int i = 0; i < 3; ++i) pb.key[i] = fdiv8((int)lround(pos[i] * P.ih[i]));
    pb.b = hash_find(hk, hv, hcap, pack_key(pb.key[0], pb.key[1], pb.key[2]));
    GlobalField f{pb, nbr, hk, hv, hcap, lay, U};
    rk4(pos, f, P, dt, &bad);
    px[q] = pos[0];
    py[q] = pos[1];
    pz[q] = pos[2];
  }
  if (bad) atomicAdd(bad_count, 1ull);
}

// ------------------------------------------------------------ pipeline B
// The grid and particle updates of Algorithms_RungeKutta_all::Do
// (src/Algorithms_RungeKutta_all.h:35-156), stage by stage, in the reference's
// expression order: stage 1 u2 = u0 + a dt 0.5, u1 = u0 + a dt 1/6; stage 2
// u2 = u0 + a dt 0.5, u1 += a dt 1/3; stage 3 u2 = u0 + a dt, u1 += a dt 1/3
// (all forced Sets); stage 4 u0 = u1 + a dt 1/6 through the non-forced Set.
__global__ void __launch_bounds__(256) k_acc_zero(const int* __restrict__ blist, int nlive,
                                                  const int8_t* __restrict__ lay, double* ax, double* ay, double* az) {
  for (int bi = blockIdx.x; bi < nlive; bi += gridDim.x) {
    size_t base = (size_t)blist[bi] * kCells;
    for (int o = threadIdx.x; o < kCells; o += blockDim.x) {
      size_t c = base + o;
      if (lay[c] == kMissing) continue;
      ax[c] = 0.0;
      ay[c] = 0.0;
      az[c] = 0.0;
    }
  }
}

struct Fields3 {
  double* f[3][3];  // speed buffers 0..2, components x..z
  double* a[3];     // acceleration
};

__global__ void __launch_bounds__(256) k_grid_stage(const int* __restrict__ blist, int nlive,
                                                    const int8_t* __restrict__ lay, const uint8_t* __restrict__ flags,
                                                    Fields3 F, const Scalars* __restrict__ ds, int stage) {
  const double dt = ds->dt;
  for (int bi = blockIdx.x; bi < nlive; bi += gridDim.x) {
    size_t base = (size_t)blist[bi] * kCells;
    for (int o = threadIdx.x; o < kCells; o += blockDim.x) {
      size_t c = base + o;
      if (lay[c] == kMissing) continue;
      const uint8_t fl = flags[c];
      for (int i = 0; i < 3; ++i) {
        const double a = F.a[i][c];
        const double u0 = F.f[0][i][c];
        if (stage == 1) {
          F.f[2][i][c] = u0 + a * dt * 0.5;
          F.f[1][i][c] = u0 + a * dt * 1. / 6.;
        } else if (stage == 2) {
          F.f[2][i][c] = u0 + a * dt * 0.5;
          F.f[1][i][c] = F.f[1][i][c] + a * dt * 1. / 3.;
        } else if (stage == 3) {
          F.f[2][i][c] = u0 + a * dt;
          F.f[1][i][c] = F.f[1][i][c] + a * dt * 1. / 3.;
        } else if (!(fl & (1u << i))) {
          F.f[0][i][c] = F.f[1][i][c] + a * dt * 1. / 6.;
        }
      }
    }
  }
}

// Policy_Move_Particle's particle updates (src/Policy_Move_Particle.h:24-56,
// the speed from Policy_Speed_Interpolation_Linear[_Symmetric]::Get_Speed of
// the stage's speed field U): stage 1 p2 = p0 + dt 0.5 v(p0), p1 = p0 + dt/6 v(p0);
// stages 2 and 3 p2 = p0 + s v(p2) (s = dt 0.5, dt), then p1 += dt/3 v(p2 new);
// stage 4 p0 = p1 + dt/6 v(p2).
struct PartBufs {
  double* p[3][3];  // positions 0..2, components x..z
};

__global__ void __launch_bounds__(256) k_particle_stage(PartBufs B, const int* __restrict__ nbr,
                                                        const unsigned long long* __restrict__ hk,
                                                        const int* __restrict__ hv, int64_t hcap,
                                                        const int8_t* __restrict__ lay, const double* __restrict__ ux,
                                                        const double* __restrict__ uy, const double* __restrict__ uz,
                                                        Params P, const Scalars* __restrict__ ds, int stage,
                                                        unsigned long long* bad_count) {
  const double dt = ds->dt;
  const int64_t n = ds->np;
  const double* U[3] = {ux, uy, uz};
  int bad = 0;
  auto speed = [&](const double* pos, double* v) {
    PBase pb;
    for (int i = 0; i < 3; ++i) pb.key[i] = fdiv8((int)lround(pos[i] * P.ih[i]));
    pb.b = hash_find(hk, hv, hcap, pack_key(pb.key[0], pb.key[1], pb.key[2]));
    GlobalField f{pb, nbr, hk, hv, hcap, lay, U};
    get_speed(pos, v, f, P, P.interp_sym, &bad);
  };
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    double p0[3], p1[3], p2[3], v[3];
    for (int i = 0; i < 3; ++i) p0[i] = B.p[0][i][q];
    if (stage == 1) {
      speed(p0, v);
      for (int i = 0; i < 3; ++i) {
        B.p[2][i][q] = p0[i] + dt * 0.5 * v[i];
        B.p[1][i][q] = p0[i] + dt * 1.0 / 6.0 * v[i];
      }
    } else if (stage == 2 || stage == 3) {
      const double s = stage == 2 ? dt * 0.5 : dt;
      for (int i = 0; i < 3; ++i) p2[i] = B.p[2][i][q];
      speed(p2, v);
      for (int i = 0; i < 3; ++i) p2[i] = p0[i] + s * v[i];
      speed(p2, v);
      for (int i = 0; i < 3; ++i) {
        B.p[2][i][q] = p2[i];
        p1[i] = B.p[1][i][q];
        B.p[1][i][q] = p1[i] + dt * 1.0 / 3.0 * v[i];
      }
    } else {
      for (int i = 0; i < 3; ++i) p2[i] = B.p[2][i][q];
      speed(p2, v);
      for (int i = 0; i < 3; ++i) B.p[0][i][q] = B.p[1][i][q] + dt * 1.0 / 6.0 * v[i];
    }
  }
  if (bad) atomicAdd(bad_count, 1ull);
}

__global__ void k_half_time(Scalars* ds) { ds->t += 0.5 * ds->dt; }

int rk_all_stage_update(Ctx* c, int stage, const double* const* U) {
  cudaStream_t st = c->stream;
  size_t cap = (size_t)c->cap_bricks * kCells;
  Fields3 F;
  for (int i = 0; i < 3; ++i) {
    F.f[0][i] = c->f64 + (size_t)(U0X + i) * cap;
    F.f[1][i] = c->f64 + (size_t)(U1X + i) * cap;
    F.f[2][i] = c->u2 + (size_t)i * cap;
    F.a[i] = c->f64 + (size_t)(AX + i) * cap;
  }
  if (c->nlive_host > 0) {
    k_grid_stage<<<c->nlive_host, 256, 0, st>>>(c->blist, c->nlive_host, c->lay, c->flags, F, c->ds, stage); MAC_COUNT(c);
  }
  if (c->np_host > 0) {
    PartBufs B;
    B.p[0][0] = c->px;
    B.p[0][1] = c->py;
    B.p[0][2] = c->pz;
    for (int k = 0; k < 2; ++k)
      for (int i = 0; i < 3; ++i) B.p[k + 1][i] = c->pbuf[k][i];
    int g = grid_for(c->np_host, 256);
    if (g > 148 * 16) g = 148 * 16;
    prof_begin(c, PH_MOVE);
    k_particle_stage<<<g, 256, 0, st>>>(B, c->nbr, c->hkeys, c->hval, c->hcap, c->lay, U[0], U[1], U[2], c->dp, c->ds,
                                        stage, &c->ds->bad_reads); MAC_COUNT(c);
    prof_end(c, PH_MOVE);
  }
  if (stage < 4 && c->nlive_host > 0) {
    k_acc_zero<<<c->nlive_host, 256, 0, st>>>(c->blist, c->nlive_host, c->lay, F.a[0], F.a[1], F.a[2]); MAC_COUNT(c);
  }
  if (stage == 1 || stage == 3) {
    k_half_time<<<1, 1, 0, st>>>(c->ds); MAC_COUNT(c);
  }
  return check(cudaGetLastError());
}

int acc_zero(Ctx* c) {
  if (c->nlive_host == 0) return MAC_OK;
  size_t cap = (size_t)c->cap_bricks * kCells;
  k_acc_zero<<<c->nlive_host, 256, 0, c->stream>>>(c->blist, c->nlive_host, c->lay, c->f64 + AX * cap,
                                                   c->f64 + AY * cap, c->f64 + AZ * cap); MAC_COUNT(c);
  return check(cudaGetLastError());
}

int bin_particles(Ctx* c, cudaStream_t st) {
  if (c->np_host == 0 || c->nlive_host == 0) return MAC_OK;
  const int64_t np = c->np_host;
  const int stray = (int)c->cap_bricks;
  int g = grid_for(np, 256);
  if (g > 148 * 16) g = 148 * 16;
  int rc = check(cudaMemsetAsync(c->bcount, 0, sizeof(int) * (c->cap_bricks + 1), st));
  if (!rc) rc = check(cudaMemsetAsync(c->bcursor, 0, sizeof(int) * (c->cap_bricks + 1) * kCells, st));
  if (rc) return rc;
  k_bin_count<<<g, 256, 0, st>>>(c->px, c->py, c->pz, np, c->dp, c->hkeys, c->hval, c->hcap, c->pbrick, c->bcursor,
                                 stray); MAC_COUNT(c);
  k_cell_scan<<<c->nlive_host + 1, kCells, 0, st>>>(c->blist, c->nlive_host, stray, c->bcursor, c->bcount); MAC_COUNT(c);
  k_bin_scan<<<1, 1024, 0, st>>>(c->bcount, c->boff, stray + 1); MAC_COUNT(c);
  k_bin_scatter<<<g, 256, 0, st>>>(c->px, c->py, c->pz, np, c->pbrick, c->boff, c->bcursor, c->px2, c->py2,
                                   c->pz2); MAC_COUNT(c);
  std::swap(c->px, c->px2);
  std::swap(c->py, c->py2);
  std::swap(c->pz, c->pz2);
  return check(cudaGetLastError());
}

int move_binned(Ctx* c) {
  if (c->np_host == 0 || c->nlive_host == 0) return MAC_OK;
  cudaStream_t st = c->stream;
  const size_t cap = (size_t)c->cap_bricks * kCells;
  const int stray = (int)c->cap_bricks;
  unsigned long long* bad = &c->ds->bad_reads;
  k_move_binned<<<c->nlive_host, 256, 0, st>>>(c->px, c->py, c->pz, c->blist, c->bkey, c->nbr, c->boff, c->hkeys,
                                               c->hval, c->hcap, c->lay, c->f64 + U0X * cap, c->f64 + U0Y * cap,
                                               c->f64 + U0Z * cap, c->dp, c->ds, bad); MAC_COUNT(c);
  k_move_stray<<<4, 256, 0, st>>>(c->px, c->py, c->pz, c->boff, stray, c->nbr, c->hkeys, c->hval, c->hcap, c->lay,
                                  c->f64 + U0X * cap, c->f64 + U0Y * cap, c->f64 + U0Z * cap, c->dp, c->ds,
                                  bad); MAC_COUNT(c);
  return check(cudaGetLastError());
}

int launch_side_binning(Ctx* c) {
  if (!c->bin_pending) return MAC_OK;
  c->bin_pending = 0;
  int rc = check(cudaEventRecord(c->ev_topo, c->stream));
  if (!rc) rc = check(cudaStreamWaitEvent(c->side, c->ev_topo, 0));
  if (!rc) rc = bin_particles(c, c->side);
  if (!rc) rc = check(cudaEventRecord(c->ev_bins, c->side));
  if (!rc) c->bin_launched = 1;
  return rc;
}

int move_particles(Ctx* c) {
  if (c->np_host == 0 || c->nlive_host == 0) return MAC_OK;
  prof_begin(c, PH_MOVE);
  int rc = bin_particles(c, c->stream);
  if (!rc) rc = move_binned(c);
  prof_end(c, PH_MOVE);
  return rc;
}

}  // namespace mac
