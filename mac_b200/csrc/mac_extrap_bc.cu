// Algorithm_Extrapolate_Boundary_Condition, 3D form
// (src/Algorithm_Extrapolate_Boundary_Condition.h:454-975; common part :52-252),
// with Policy_Is_In_Domain_Speed (src/Policy_Is_In_Domain_Speed.h:15-48): the
// boundary conditions of the speed field at the free surface, written into
// the air-side faces of the boundary cells (fluid cells with an air face
// neighbour). The reference composes it at output time
// (test/Lateral_jet_3.cpp:706-711).
//
// Order. The reference visits its hash map in iteration order and a boundary
// cell's case writes faces that later cells read. The device fixes the order:
// boundary cells by colour (key x, y, z mod 5), colours in turn, the cells of
// one colour at once. Every read and write of one cell's case lies within
// Chebyshev distance 2 of it, so cells of one colour (5 or more apart on some
// axis) never touch a common face and the result equals the sequential visit
// in colour order; the three-face corners run after all other cases, colours
// in reverse (the reference unwinds them from a stack). The oracle's
// alg_extrap_bc (command extrapbc) visits in the same order and the device
// matches it bit for bit (no contraction in this file).
//
// Reference details kept: GetNeighbour(i, 0) is the -e_i neighbour (the
// neighbour tables index (s + 1) >> 1, src/Offset_GetNeighbour.h:52-57), so
// apply_nan_extrap counts it twice; Apply_Div_3d keeps the last tangential
// term of its loop; the n == 1 case's flag b is never cleared. An air or
// missing neighbour counts as no boundary where the reference reads an unset
// counter; a read of a missing cell gives NaN, a write to one is dropped.
// Every write goes through the non-forced Set (const faces keep their value,
// src/Data_Grid_Speed.tpp:19-26). The 3x3 corner systems (the reference's
// Umfpack policy) are solved by Gaussian elimination with partial pivoting.
#include <cmath>
#include <vector>

#include "mac_internal.cuh"

namespace mac {

#define EB_CUDA(x)                      \
  do {                                  \
    const int rc_ = check(x);           \
    if (rc_ != MAC_OK) return rc_;      \
  } while (0)

constexpr int kEbColors = 125;

struct EbView {
  const int* nbr;
  const int* bkey;
  const int8_t* lay;
  const uint8_t* type;
  const uint8_t* flags;
  double* u[3];
  double ih[3], h[3];
};

__device__ inline double eb_nan() { return __longlong_as_double(0x7ff8000000000000ll); }
__device__ inline bool eb_isnan(double v) { return v != v; }

// A cell as (brick b, local x y z) of brick b; local coordinates may leave
// [0, 8) by up to 8 (the 27-brick table).
struct EbCell {
  int b, x, y, z;
};
__device__ inline int64_t eb_index(const EbView& V, EbCell k) {
  const int dx = k.x < 0 ? -1 : (k.x >= 8 ? 1 : 0), dy = k.y < 0 ? -1 : (k.y >= 8 ? 1 : 0),
            dz = k.z < 0 ? -1 : (k.z >= 8 ? 1 : 0);
  const int nb = (dx | dy | dz) == 0 ? k.b : V.nbr[(size_t)k.b * kNbr + nbr_index(dx, dy, dz)];
  if (nb < 0) return -1;
  const int64_t c = (int64_t)nb * kCells + (k.x - 8 * dx) + 8 * (k.y - 8 * dy) + 64 * (k.z - 8 * dz);
  return V.lay[c] == kMissing ? -1 : c;
}
__device__ inline EbCell eb_nb(EbCell k, int i, int s) {  // i 1..3, s = 0 means -1
  const int d = s > 0 ? 1 : -1;
  if (i == 1) k.x += d;
  else if (i == 2) k.y += d;
  else k.z += d;
  return k;
}
__device__ inline bool eb_air_at(const EbView& V, int64_t c) {  // GetIsAir: air and solid
  return c < 0 || !(V.type[c] == MAC_CELL_FLUID || V.type[c] == MAC_CELL_INFLOW || V.type[c] == MAC_CELL_INTERIOR);
}
__device__ inline double eb_u(const EbView& V, EbCell k, int i) {
  const int64_t c = eb_index(V, k);
  return c < 0 ? eb_nan() : V.u[i - 1][c];
}
__device__ inline void eb_set(const EbView& V, EbCell k, int i, double v) {
  const int64_t c = eb_index(V, k);
  if (c >= 0 && !(V.flags[c] & (1u << (i - 1)))) V.u[i - 1][c] = v;
}
// IsBoundary (:89-119): the air face neighbours in (i, s) order; 0 for air or missing
__device__ inline int eb_boundary(const EbView& V, EbCell k, int* dir, int* sign) {
  const int64_t c = eb_index(V, k);
  if (c < 0 || eb_air_at(V, c)) return 0;
  int n = 0;
  for (int i = 1; i <= 3; ++i)
    for (int s = -1; s <= 1; s += 2) {
      const int64_t c2 = eb_index(V, eb_nb(k, i, s));
      if (c2 >= 0 && eb_air_at(V, c2)) {
        dir[n] = i;
        sign[n] = s;
        ++n;
      }
    }
  return n;
}
__device__ inline bool eb_in_domain(const EbView& V, EbCell k, int d) {  // Get_Is_Speed_In_Domain
  const EbCell k2 = eb_nb(k, d, -1);
  const int64_t c2 = eb_index(V, k2);
  const bool f1 = !eb_air_at(V, eb_index(V, k));
  if (c2 < 0) return f1;
  const bool f2 = !eb_air_at(V, c2);
  if (f1 && f2) return true;
  if (!f1 && !f2) return false;
  const int64_t c3 = eb_index(V, f1 ? eb_nb(k, d, 1) : eb_nb(k2, d, -1));
  if (c3 < 0) return true;
  return eb_air_at(V, c3);
}
__device__ void eb_div(const EbView& V, EbCell k, int d, int sign) {  // Apply_Div_3d (:912-932)
  EbCell n = eb_nb(k, d, 1);
  double v = eb_u(V, k, d);
  if (sign == -1) {
    v = eb_u(V, n, d);
    n = k;
  }
  double res = 0;
  for (int d2 = 1; d2 <= 3; ++d2) {
    if (d2 == d) continue;
    res = V.ih[d2 - 1] * (eb_u(V, eb_nb(k, d2, 1), d2) - eb_u(V, k, d2));
  }
  res = v - sign * res * V.h[d - 1];
  eb_set(V, n, d, res);
}
__device__ void eb_plane(const EbView& V, EbCell a, EbCell b, int d, int sign, int d2) {  // Apply_3d_Plane (:897-911)
  EbCell n = a, n2 = b;
  if (sign == 1) {
    n = eb_nb(a, d, 1);
    n2 = eb_nb(b, d, 1);
  }
  const double v1 = eb_u(V, n, d), v2 = eb_u(V, n2, d), v3 = eb_u(V, b, d2);
  const double v = -sign * V.ih[d2 - 1] * V.h[d - 1] * (v2 - v1) + v3;
  eb_set(V, eb_nb(b, d, sign), d2, v);
}
__device__ void eb_plane45(const EbView& V, EbCell k, int sa, int da, int sb, int db) {  // Apply_3d_Plane_45 (:934-952)
  EbCell n1 = eb_nb(k, da, 1), n2 = eb_nb(k, db, 1);
  double v1 = eb_u(V, k, da), v2 = eb_u(V, k, db);
  if (sa == -1) {
    v1 = eb_u(V, n1, da);
    n1 = k;
  }
  if (sb == -1) {
    v2 = eb_u(V, n2, db);
    n2 = k;
  }
  eb_set(V, n1, da, v1);
  eb_set(V, n2, db, v2);
}

// Step 1, apply_set_nan (:149-177) on every existing air cell of the live bricks.
__global__ void __launch_bounds__(512) k_eb_set_nan(const int* __restrict__ blist, EbView V) {
  const int b = blist[blockIdx.x];
  const EbCell k{b, (int)(threadIdx.x & 7), (int)((threadIdx.x >> 3) & 7), (int)(threadIdx.x >> 6)};
  const int64_t c = (int64_t)b * kCells + threadIdx.x;
  if (V.lay[c] == kMissing || !eb_air_at(V, c)) return;
  for (int i = 1; i <= 3; ++i)
    for (int s = -1; s <= 1; s += 2) {
      const EbCell k2 = eb_nb(k, i, s);
      const int64_t c2 = eb_index(V, k2);
      if (c2 >= 0) {
        if (eb_air_at(V, c2)) eb_set(V, s == -1 ? k : k2, i, eb_nan());
      } else if (s == -1) {
        eb_set(V, k, i, eb_nan());
      }
    }
}

__device__ inline int eb_mod5(int v) { return ((v % 5) + 5) % 5; }
__device__ inline int eb_color(const EbView& V, EbCell k) {
  return eb_mod5(V.bkey[3 * k.b] * 8 + k.x) + 5 * eb_mod5(V.bkey[3 * k.b + 1] * 8 + k.y) +
         25 * eb_mod5(V.bkey[3 * k.b + 2] * 8 + k.z);
}

// Boundary cells per colour: MODE 0 counts, MODE 1 writes each cell's pool
// index into its colour's run (cursor[] starts at the runs' offsets).
template <int MODE>
__global__ void __launch_bounds__(512) k_eb_bin(const int* __restrict__ blist, EbView V, int* count, int* cursor,
                                                int* list) {
  const int b = blist[blockIdx.x];
  const EbCell k{b, (int)(threadIdx.x & 7), (int)((threadIdx.x >> 3) & 7), (int)(threadIdx.x >> 6)};
  int dir[6], sign[6];
  if (eb_boundary(V, k, dir, sign) == 0) return;
  const int col = eb_color(V, k);
  if (MODE == 0) atomicAdd(&count[col], 1);
  else list[atomicAdd(&cursor[col], 1)] = b * kCells + (int)threadIdx.x;
}

__device__ inline EbCell eb_cell_of(int idx) {
  const int o = idx & 511;
  return EbCell{idx >> 9, o & 7, (o >> 3) & 7, o >> 6};
}

// Step 2, Choose_Boundary_Case_3d (:793-890) for one colour's cells, the
// three-face corners left to step 3.
__global__ void __launch_bounds__(128) k_eb_choose(const int* __restrict__ list, int n, EbView V) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const EbCell k = eb_cell_of(list[t]);
  int dir[6], sign[6];
  const int nn = eb_boundary(V, k, dir, sign);
  if (nn == 1) {
    eb_div(V, k, dir[0], sign[0]);
    for (int d2 = 1; d2 <= 3; ++d2) {
      if (d2 == dir[0]) continue;
      for (int i = -1; i <= 1; i += 2) {
        const EbCell k2 = eb_nb(k, d2, i);
        int dt[6], st[6];
        const int nt = eb_boundary(V, k2, dt, st);
        if (nt == 1) eb_div(V, k2, dt[0], st[0]);
        if (nt == 1 && dt[0] == dir[0]) {
          if (i < 0) eb_plane(V, k2, k, dir[0], sign[0], d2);
          else eb_plane(V, k, k2, dir[0], sign[0], d2);
        }
      }
      const EbCell k3 = sign[0] == 1 ? eb_nb(k, dir[0], 1) : k;
      if (!eb_in_domain(V, k, dir[0])) eb_set(V, k3, dir[0], eb_nan());
    }
  } else if (nn == 2) {
    if (dir[0] != dir[1]) eb_plane45(V, k, sign[0], dir[0], sign[1], dir[1]);
  } else if (nn != 3) {
    for (int i = 0; i < nn; ++i) {
      const EbCell k2 = sign[i] == 1 ? eb_nb(k, dir[i], 1) : k;
      if (!eb_in_domain(V, k2, dir[i])) eb_set(V, k2, dir[i], eb_nan());
    }
  }
}

// A x = b, A row-major: Gaussian elimination with partial pivoting (rows swap
// on a strictly larger |pivot|), then back substitution.
__device__ inline void eb_solve3(const double* A, const double* b, double* x) {
  double m[3][4];
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) m[r][c] = A[3 * r + c];
    m[r][3] = b[r];
  }
  for (int c = 0; c < 3; ++c) {
    int p = c;
    for (int r = c + 1; r < 3; ++r)
      if (fabs(m[r][c]) > fabs(m[p][c])) p = r;
    if (p != c)
      for (int j = 0; j < 4; ++j) {
        const double t = m[c][j];
        m[c][j] = m[p][j];
        m[p][j] = t;
      }
    for (int r = c + 1; r < 3; ++r) {
      const double f = m[r][c] / m[c][c];
      for (int j = c; j < 4; ++j) m[r][j] = m[r][j] - f * m[c][j];
    }
  }
  for (int r = 2; r >= 0; --r) {
    double v = m[r][3];
    for (int j = r + 1; j < 3; ++j) v = v - m[r][j] * x[j];
    x[r] = v / m[r][r];
  }
}

// Step 3, SolveMatrix (:571-775) for one colour's three-face corners: the 3x3
// system of CreateMatrix (:551-570; CSC value[3 j + r] = A[r][j]) with the
// right-hand side of the reference's terms in their order.
__global__ void __launch_bounds__(128) k_eb_corner(const int* __restrict__ list, int n, EbView V) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const EbCell k = eb_cell_of(list[t]);
  int dir[6], sign[6];
  const int nn = eb_boundary(V, k, dir, sign);
  if (nn != 3) return;
  int sg[3] = {0, 0, 0};
  for (int a = 1; a <= 3; ++a)
    for (int i = 0; i < nn; ++i)
      if (dir[i] == a) {
        sg[a - 1] = sign[i];
        break;
      }
  if (sg[0] == 0 || sg[1] == 0 || sg[2] == 0) return;
  const int s1 = sg[0], s2 = sg[1], s3 = sg[2];
  const double* ih = V.ih;
  const double A[9] = {
      -s1 * 2 * ih[0] - s1 * 0.5 * ih[2], s2 * 2 * ih[1] + s2 * 0.5 * ih[2], -s3 * 0.5 * ih[0] + s2 * s3 * 0.5 * ih[1],
      -s1 * 0.5 * ih[2] + s1 * 0.5 * ih[1], s2 * 2 * ih[1] + s2 * 0.5 * ih[1], -s3 * 2 * ih[2] - s3 * 0.5 * ih[0],
      s1 * ih[0], s2 * ih[1], s3 * ih[2]};
  const EbCell e1 = eb_nb(k, 1, 1), e2 = eb_nb(k, 2, 1), e3 = eb_nb(k, 3, 1);
  const EbCell m1 = eb_nb(k, 1, -s1), m2 = eb_nb(k, 2, -s2), m3 = eb_nb(k, 3, -s3);
  double b[3], x[3];
  b[0] = 0;
  b[0] += s1 == 1 ? -2 * ih[0] * eb_u(V, k, 1) : 2 * ih[0] * eb_u(V, e1, 1);
  b[0] += s2 == 1 ? 2 * ih[1] * eb_u(V, k, 2) : -2 * ih[1] * eb_u(V, e2, 2);
  b[0] += s3 == 1 ? 0.5 * ih[0] * eb_u(V, k, 3) : -0.5 * ih[0] * eb_u(V, e3, 3);
  b[0] += s3 * 0.5 * ih[0] * (-eb_u(V, m1, 3) - eb_u(V, eb_nb(m1, 3, 1), 3));
  b[0] += s1 == 1 ? 0.5 * ih[2] * eb_u(V, k, 1) : -0.5 * ih[2] * eb_u(V, e1, 1);
  b[0] += s1 * 0.5 * ih[2] * (-eb_u(V, m3, 1) - eb_u(V, eb_nb(m3, 1, 1), 1));
  b[0] += s3 == 1 ? -0.5 * ih[1] * eb_u(V, k, 3) : 0.5 * ih[1] * eb_u(V, e3, 3);
  b[0] += s3 * 0.5 * ih[1] * (eb_u(V, m2, 3) + eb_u(V, eb_nb(m2, 3, 1), 3));
  b[0] += s2 == 1 ? -0.5 * ih[2] * eb_u(V, k, 2) : 0.5 * ih[2] * eb_u(V, e2, 2);
  b[0] += s2 * 0.5 * ih[2] * (eb_u(V, m3, 2) + eb_u(V, eb_nb(m3, 2, 1), 2));
  b[1] = 0;
  b[1] += s3 == 1 ? -2 * ih[2] * eb_u(V, k, 3) : 2 * ih[2] * eb_u(V, m3, 3);
  b[1] += s2 == 1 ? 2 * ih[1] * eb_u(V, k, 2) : -2 * ih[1] * eb_u(V, e2, 2);
  b[1] += s3 == 1 ? 0.5 * ih[0] * eb_u(V, k, 3) : -0.5 * ih[0] * eb_u(V, e3, 3);
  b[1] += s3 * 0.5 * ih[0] * (-eb_u(V, m1, 3) - eb_u(V, eb_nb(m1, 3, 1), 3));
  b[1] += s1 == 1 ? 0.5 * ih[2] * eb_u(V, k, 1) : -0.5 * ih[2] * eb_u(V, e1, 1);
  b[1] += s1 * 0.5 * ih[2] * (-eb_u(V, m3, 1) - eb_u(V, eb_nb(m3, 1, 1), 1));
  b[1] += s1 == 1 ? -0.5 * ih[1] * eb_u(V, k, 1) : -0.5 * ih[1] * eb_u(V, e1, 1);
  b[1] += s1 * 0.5 * ih[1] * (eb_u(V, m2, 1) + eb_u(V, eb_nb(m2, 1, 1), 1));
  b[1] += s2 == 1 ? -0.5 * ih[0] * eb_u(V, k, 2) : 0.5 * ih[0] * eb_u(V, e2, 2);
  b[1] += s2 * 0.5 * ih[0] * (eb_u(V, m1, 2) + eb_u(V, eb_nb(m1, 2, 1), 2));
  b[2] = 0;
  b[2] += s1 == 1 ? ih[0] * eb_u(V, k, 1) : -ih[0] * eb_u(V, e1, 1);
  b[2] += s2 == 1 ? ih[1] * eb_u(V, k, 2) : -ih[1] * eb_u(V, e2, 2);
  b[2] += s3 == 1 ? ih[2] * eb_u(V, k, 3) : -ih[2] * eb_u(V, e3, 3);
  if (!eb_isnan(b[0]) && !eb_isnan(b[1]) && !eb_isnan(b[2])) {
    eb_solve3(A, b, x);
  } else {
    x[0] = x[1] = x[2] = eb_nan();
  }
  eb_set(V, s1 == 1 ? e1 : k, 1, x[0]);
  eb_set(V, s2 == 1 ? e2 : k, 2, x[1]);
  eb_set(V, s3 == 1 ? e3 : k, 3, x[2]);
}

// Step 4, apply_nan_extrap (:183-251) for one colour's boundary cells.
__global__ void __launch_bounds__(128) k_eb_nan_extrap(const int* __restrict__ list, int n, EbView V) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const EbCell k = eb_cell_of(list[t]);
  int tab[2][6], nn = 0;
  for (int i = 1; i <= 3; ++i) {
    if (eb_isnan(eb_u(V, k, i))) {
      tab[0][nn] = i;
      tab[1][nn] = 0;
      ++nn;
    }
    if (eb_isnan(eb_u(V, eb_nb(k, i, 1), i))) {
      tab[0][nn] = i;
      tab[1][nn] = 1;
      ++nn;
    }
  }
  if (nn == 0) return;
  for (int j = 0; j < nn; ++j) {
    const int d = tab[0][j];
    const EbCell k2 = tab[1][j] == 1 ? eb_nb(k, d, 1) : k;
    double vt = 0;
    int cnt = 0;
    for (int d2 = 1; d2 <= 3; ++d2)
      for (int s = -1; s <= 1; ++s) {
        const double add = eb_u(V, eb_nb(k2, d2, s), d);
        if (!eb_isnan(add)) {
          vt += add;
          ++cnt;
        }
      }
    if (cnt != 0) vt /= cnt;
    eb_set(V, k2, d, vt);
  }
  double div = 0;
  for (int i = 1; i <= 3; ++i) div += V.ih[i - 1] * (eb_u(V, eb_nb(k, i, 1), i) - eb_u(V, k, i));
  const double cor = div / nn;
  for (int j = 0; j < nn; ++j) {
    const int d = tab[0][j], sg = tab[1][j];
    const EbCell k2 = sg == 1 ? eb_nb(k, d, 1) : k;
    eb_set(V, k2, d, eb_u(V, k2, d) - (2 * sg - 1) * V.h[d - 1] * cor);
  }
}

// The whole algorithm on speed buffer ispeed. Scratch: the boundary-cell list
// in the solver vector q (one int per cell slot), colour counts and cursors in
// the context's small work array.
int extrapolate_boundary_condition(Ctx* c, int ispeed) {
  const int nlive = c->nlive_host;
  if (nlive == 0) return MAC_OK;
  cudaStream_t st = c->stream;
  const size_t cap = (size_t)c->cap_bricks * kCells;
  EbView V;
  V.nbr = c->nbr;
  V.bkey = c->bkey;
  V.lay = c->lay;
  V.type = c->type;
  V.flags = c->flags;
  for (int i = 0; i < 3; ++i) {
    V.u[i] = c->f64 + (size_t)(U0X + 3 * ispeed + i) * cap;
    V.h[i] = c->dp.h[i];
    V.ih[i] = c->dp.ih[i];
  }
  if (!c->eb_work) {
    int rc = check(cudaMalloc((void**)&c->eb_work, sizeof(int) * 2 * kEbColors));
    if (rc) return rc;
  }
  int* count = c->eb_work;
  int* cursor = c->eb_work + kEbColors;
  int* list = (int*)c->q;
  k_eb_set_nan<<<nlive, 512, 0, st>>>(c->blist, V); MAC_COUNT(c);
  EB_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * kEbColors, st));
  k_eb_bin<0><<<nlive, 512, 0, st>>>(c->blist, V, count, cursor, list); MAC_COUNT(c);
  int hc[kEbColors], off[kEbColors + 1];
  EB_CUDA(cudaMemcpyAsync(hc, count, sizeof(hc), cudaMemcpyDeviceToHost, st));
  EB_CUDA(cudaStreamSynchronize(st));
  off[0] = 0;
  for (int i = 0; i < kEbColors; ++i) off[i + 1] = off[i] + hc[i];
  EB_CUDA(cudaMemcpyAsync(cursor, off, sizeof(int) * kEbColors, cudaMemcpyHostToDevice, st));
  k_eb_bin<1><<<nlive, 512, 0, st>>>(c->blist, V, count, cursor, list); MAC_COUNT(c);
  for (int col = 0; col < kEbColors; ++col)
    if (hc[col]) {
      k_eb_choose<<<grid_for(hc[col], 128), 128, 0, st>>>(list + off[col], hc[col], V); MAC_COUNT(c);
    }
  for (int col = kEbColors - 1; col >= 0; --col)
    if (hc[col]) {
      k_eb_corner<<<grid_for(hc[col], 128), 128, 0, st>>>(list + off[col], hc[col], V); MAC_COUNT(c);
    }
  for (int col = 0; col < kEbColors; ++col)
    if (hc[col]) {
      k_eb_nan_extrap<<<grid_for(hc[col], 128), 128, 0, st>>>(list + off[col], hc[col], V); MAC_COUNT(c);
    }
  // the copy of off[] must not outlive this frame
  EB_CUDA(cudaStreamSynchronize(st));
  return check(cudaGetLastError());
}

}  // namespace mac

extern "C" int mac_extrapolate_boundary_condition(void* ctx, int ispeed) {
  mac::Ctx* c = (mac::Ctx*)ctx;
  if (!c || ispeed < 0 || ispeed > 1) return MAC_ERR_INVALID;
  cudaSetDevice(c->prm.device);
  int rc = mac::read_scalars(c);
  return rc ? rc : mac::extrapolate_boundary_condition(c, ispeed);
}
