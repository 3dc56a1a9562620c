// Advection stage on the brick grid: gravity + first-order upwind convection
// fused with the SSP-RK2 stage updates, air-layer velocity extrapolation and
// the RK4 particle move through the staggered trilinear field.
//
// The library is compiled with -fmad=false and every expression keeps the
// reference's operation order, so these kernels reproduce the reference's
// FP64 results bit for bit from the same input state.
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

struct Fields {
  const double* u[3];  // speed buffer read by the stencil
};

// Get_Speed_At_Bound (src/Policy_Speed_Interpolation_Linear_Symmetric.h:120-127,
// identical in src/Policy_Speed_Interpolation_Linear.h:107-114).
__device__ inline double speed_at_bound(const double* const* U, const int* sn, int x, int y, int z, int i, int j) {
  int c[3] = {x, y, z};
  if (i == j) return rdv(U[j], cidx(sn, x, y, z));
  int cj[3] = {x, y, z}, ci[3] = {x, y, z}, cij[3] = {x, y, z};
  cj[j] += 1;
  ci[i] -= 1;
  cij[i] -= 1;
  cij[j] += 1;
  double a = rdv(U[j], cidx(sn, c[0], c[1], c[2]));
  double b = rdv(U[j], cidx(sn, cj[0], cj[1], cj[2]));
  double d = rdv(U[j], cidx(sn, ci[0], ci[1], ci[2]));
  double e = rdv(U[j], cidx(sn, cij[0], cij[1], cij[2]));
  return 0.25 * (((a + b) + d) + e);
}

// Policy_Upwind_1_Order::Get_Convection_Speed(neigh, i) (src/Policy_Upwind_1_Order.h:18-38,58-66).
__device__ inline double convection(const double* const* U, const int* sn, int x, int y, int z, int i,
                                    const Params& P) {
  double ret = 0;
  double U1 = rdv(U[i], cidx(sn, x, y, z));
  for (int j = 0; j < 3; ++j) {
    double Ub = speed_at_bound(U, sn, x, y, z, i, j);
    int m[3] = {x, y, z};
    if (Ub > 0) {
      m[j] -= 1;
      double U2 = rdv(U[i], cidx(sn, m[0], m[1], m[2]));
      Ub *= (U1 - U2) * P.ih[j];
    } else {
      m[j] += 1;
      double U2 = rdv(U[i], cidx(sn, m[0], m[1], m[2]));
      Ub *= (U2 - U1) * P.ih[j];
    }
    ret -= Ub;
  }
  return ret;
}

// Acceleration of face i of cell (x,y,z): forced zero, then Policy_Gravity and
// Policy_Upwind_1_Order applied through the non-forced Set (const faces keep 0).
// Gravity applies if the cell is fluid, or has a layer and its -e_g neighbour
// is fluid (src/Policy_Gravity.h:14-34); convection uses the same rule on axis
// i (src/Policy_Convection_Apply_If.h:41-61).
__device__ inline double face_accel(const double* const* U, const int* sn, const int8_t* __restrict__ lay,
                                    const uint8_t* __restrict__ type, int64_t c, uint8_t fl, int x, int y, int z,
                                    int i, const Params& P) {
  if (fl & (1u << i)) return 0.0;
  bool fluid = is_fluid(type[c]);
  bool apply = fluid;
  if (!fluid && lay[c] != kEmpty) {
    int m[3] = {x, y, z};
    m[i] -= 1;
    int64_t n = cidx(sn, m[0], m[1], m[2]);
    apply = n >= 0 && lay[n] != kMissing && is_fluid(type[n]);
  }
  double a = 0.0;
  if (i == P.gaxis) {
    bool g = fluid;
    if (!fluid && lay[c] != kEmpty) {
      int m[3] = {x, y, z};
      m[i] -= 1;
      int64_t n = cidx(sn, m[0], m[1], m[2]);
      g = n >= 0 && lay[n] != kMissing && is_fluid(type[n]);
    }
    if (g) a = a + P.g;
  }
  if (apply) a = a + convection(U, sn, x, y, z, i, P);
  return a;
}

// mode 0: acc = forces(u[ib]); mode 1: RK stage 1 (src/Algorithms_RungeKutta_RK2_TVD.h:31-43):
// u1 = u0 + a(u0)*dt, forced; mode 2: stage 2 (:45-58 after the first projection):
// acc = a(u1) and u0 = 0.5*u0 + 0.5*u1 + 0.5*acc*dt through the non-forced Set.
template <int MODE>
__global__ void __launch_bounds__(256) k_forces(const int* __restrict__ blist, int nlive, const int* __restrict__ nbr,
                                                const int8_t* __restrict__ lay, const uint8_t* __restrict__ type,
                                                const uint8_t* __restrict__ flags, double* f64, size_t cap,
                                                int ib, Params P, const Scalars* __restrict__ ds) {
  __shared__ int sn[kNbr];
  const double dt = ds->dt;
  const double* U[3];
  for (int i = 0; i < 3; ++i) U[i] = f64 + (size_t)((MODE == 2 ? 1 : (MODE == 1 ? 0 : ib)) * 3 + i) * cap;
  for (int bi = blockIdx.x; bi < nlive; bi += gridDim.x) {
    int b = blist[bi];
    if (threadIdx.x < kNbr) sn[threadIdx.x] = nbr[(size_t)b * kNbr + threadIdx.x];
    __syncthreads();
    for (int o = threadIdx.x; o < kCells; o += blockDim.x) {
      int64_t c = (int64_t)b * kCells + o;
      if (lay[c] == kMissing) continue;
      int x = o & 7, y = (o >> 3) & 7, z = o >> 6;
      uint8_t fl = flags[c];
      double a[3];
      for (int i = 0; i < 3; ++i) a[i] = face_accel(U, sn, lay, type, c, fl, x, y, z, i, P);
      if (MODE == 0) {
        for (int i = 0; i < 3; ++i) f64[(size_t)(AX + i) * cap + c] = a[i];
      } else if (MODE == 1) {
        for (int i = 0; i < 3; ++i)
          f64[(size_t)(U1X + i) * cap + c] = f64[(size_t)(U0X + i) * cap + c] + a[i] * dt;
      } else {
        for (int i = 0; i < 3; ++i) {
          f64[(size_t)(AX + i) * cap + c] = a[i];
          if (!(fl & (1u << i))) {
            double u0 = f64[(size_t)(U0X + i) * cap + c], u1 = f64[(size_t)(U1X + i) * cap + c];
            f64[(size_t)(U0X + i) * cap + c] = 0.5 * u0 + 0.5 * u1 + 0.5 * a[i] * dt;
          }
        }
      }
    }
    __syncthreads();
  }
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

__global__ void __launch_bounds__(256) k_extrapolate(const int* __restrict__ blist, int nlive, const int* __restrict__ nbr,
                                                     const int8_t* __restrict__ lay, const uint8_t* __restrict__ flags,
                                                     double* f64, size_t cap, int L) {
  __shared__ int sn[kNbr];
  for (int bi = blockIdx.x; bi < nlive; bi += gridDim.x) {
    int b = blist[bi];
    if (threadIdx.x < kNbr) sn[threadIdx.x] = nbr[(size_t)b * kNbr + threadIdx.x];
    __syncthreads();
    for (int o = threadIdx.x; o < kCells; o += blockDim.x) {
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
        const double* Ui = f64 + (size_t)(U0X + i) * cap;
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
        f64[(size_t)(U0X + i) * cap + c] = val / n;
      }
    }
    __syncthreads();
  }
}

int extrapolate(Ctx* c) {
  if (c->nlive_host == 0) return MAC_OK;
  size_t cap = (size_t)c->cap_bricks * kCells;
  prof_begin(c, PH_EXTRAPOLATE);
  for (int L = 1; L <= c->dp.layer_max + 1; ++L) {
    k_extrapolate<<<c->nlive_host, 256, 0, c->stream>>>(c->blist, c->nlive_host, c->nbr, c->lay, c->flags, c->f64,
                                                        cap, L); MAC_COUNT(c);
  }
  prof_end(c, PH_EXTRAPOLATE);
  return check(cudaGetLastError());
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

__device__ inline void get_speed(const double* pos, double* out, const PBase& pb, const int* nbr,
                                 const unsigned long long* hk, const int* hv, int64_t hcap, const int8_t* lay,
                                 const double* const* U, const Params& P, int sym, int* bad) {
  double pd[3];
  int k0[3];
  for (int i = 0; i < 3; ++i) {
    pd[i] = pos[i] * P.ih[i];
    k0[i] = (int)lround(pd[i]);
    pd[i] -= k0[i];
  }
  for (int k = 0; k < 3; ++k) {
    if (!sym) pd[k] += 0.5;
    int key[3];
    double d[3];
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
    for (int n = 0; n < 8; ++n) {
      int64_t ci = pcell(pb, nbr, hk, hv, hcap, key[0] + (n >> 2), key[1] + ((n >> 1) & 1), key[2] + (n & 1));
      if (ci < 0 || lay[ci] == kMissing) *bad = 1;
      u[n] = ci < 0 ? 0.0 : U[k][ci];
    }
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

// Algorithms_Move_Particles::Do + Policy_Advance_Ode_RungeKutta::AdvanceSolveODE
// (src/Algorithms_Move_Particles.h:29-32, src/Policy_Advance_ODE_RungeKutta.h:15-27).
__global__ void __launch_bounds__(256) k_move(double* px, double* py, double* pz, int64_t np, const int* __restrict__ nbr,
                                              const unsigned long long* __restrict__ hk, const int* __restrict__ hv,
                                              int64_t hcap, const int8_t* __restrict__ lay, const double* __restrict__ ux,
                                              const double* __restrict__ uy, const double* __restrict__ uz, Params P,
                                              const Scalars* __restrict__ ds, unsigned long long* bad_count) {
  const double dt = ds->dt;
  const double* U[3] = {ux, uy, uz};
  int bad = 0;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < np; q += (int64_t)gridDim.x * blockDim.x) {
    double pos[3] = {px[q], py[q], pz[q]};
    PBase pb;
    for (int i = 0; i < 3; ++i) pb.key[i] = fdiv8((int)lround(pos[i] * P.ih[i]));
    pb.b = hash_find(hk, hv, hcap, pack_key(pb.key[0], pb.key[1], pb.key[2]));
    double res[3], k[3], a[3], v[3];
    for (int i = 0; i < 3; ++i) res[i] = pos[i];
    get_speed(pos, v, pb, nbr, hk, hv, hcap, lay, U, P, P.interp_sym, &bad);
    for (int i = 0; i < 3; ++i) {
      k[i] = dt * v[i];
      res[i] += (1. / 6.) * k[i];
    }
    for (int i = 0; i < 3; ++i) a[i] = pos[i] + k[i] * 0.5;
    get_speed(a, v, pb, nbr, hk, hv, hcap, lay, U, P, P.interp_sym, &bad);
    for (int i = 0; i < 3; ++i) {
      k[i] = dt * v[i];
      res[i] += (1. / 3.) * k[i];
    }
    for (int i = 0; i < 3; ++i) a[i] = pos[i] + k[i] * 0.5;
    get_speed(a, v, pb, nbr, hk, hv, hcap, lay, U, P, P.interp_sym, &bad);
    for (int i = 0; i < 3; ++i) {
      k[i] = dt * v[i];
      res[i] += (1. / 3.) * k[i];
    }
    for (int i = 0; i < 3; ++i) a[i] = pos[i] + k[i];
    get_speed(a, v, pb, nbr, hk, hv, hcap, lay, U, P, P.interp_sym, &bad);
    for (int i = 0; i < 3; ++i) {
      k[i] = dt * v[i];
      res[i] += (1. / 6.) * k[i];
    }
    px[q] = res[0];
    py[q] = res[1];
    pz[q] = res[2];
  }
  if (bad) atomicAdd(bad_count, 1ull);
}

int move_particles(Ctx* c) {
  if (c->np_host == 0) return MAC_OK;
  size_t cap = (size_t)c->cap_bricks * kCells;
  int g = grid_for(c->np_host, 256);
  if (g > 148 * 16) g = 148 * 16;
  unsigned long long* bad = &c->ds->bad_reads;
  prof_begin(c, PH_MOVE);
  k_move<<<g, 256, 0, c->stream>>>(c->px, c->py, c->pz, c->np_host, c->nbr, c->hkeys, c->hval, c->hcap, c->lay,
                                   c->f64 + U0X * cap, c->f64 + U0Y * cap, c->f64 + U0Z * cap, c->dp, c->ds, bad); MAC_COUNT(c);
  prof_end(c, PH_MOVE);
  return check(cudaGetLastError());
}

}  // namespace mac
