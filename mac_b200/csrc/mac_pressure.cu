// Pressure projection on the brick grid: Algorithms_Solve_Pressure
// (src/Algorithms_Solve_Pressure.h:44-222) with Policy_Divergence,
// Policy_Gradiant, Policy_Von_Neumann_Boundary and Policy_Pressure_If_Correction,
// solving the same ghost-fluid system the reference assembles for Umfpack, but
// matrix-free and iteratively:
//
//   A p = div u,  A = 7-point Laplacian over in-domain cells; per face of an
//   in-domain cell c: missing neighbour or non-domain neighbour -> Dirichlet
//   (p = 0, diagonal only); const face -> Neumann (nothing); in-domain
//   neighbour -> coupling 1/h^2.
//
// We solve M x = -div u with M = -A (symmetric positive definite) by CG in
// FP64 with the multigrid preconditioner of mac_mg.cu (FP64 storage for the
// plain form, FP32 for the mixed form) or Jacobi. The CG recurrences, dot
// products and the final divergence check are always FP64. Vector kernels run
// one 512-thread block per brick that holds an in-domain cell; per-block
// partial sums are added in a fixed order.
#include <cstdio>
#include <cstring>
#include <utility>

#include <vector>

#include "mac_internal.cuh"
#include "mac_unet.cuh"

namespace mac {

// ------------------------------------------------------------ allocation
template <class T>
static int dalloc(T** p, size_t n) {
  return check(cudaMalloc((void**)p, sizeof(T) * (n ? n : 1)));
}

int alloc_solver(Ctx* c) {
  size_t nc = (size_t)c->cap_bricks * kCells;
  int rc = MAC_OK;
  auto A = [&](int r) { if (rc == MAC_OK) rc = r; };
  A(dalloc(&c->fmask, nc));
  A(dalloc(&c->x, nc));
  A(dalloc(&c->b, nc));
  A(dalloc(&c->r, nc));
  A(dalloc(&c->r2, nc));
  A(dalloc(&c->z, nc));
  A(dalloc(&c->pd, nc));
  A(dalloc(&c->pd2, nc));
  A(dalloc(&c->q, nc));
  A(dalloc(&c->dbl, c->cap_bricks));
  A(dalloc(&c->drow, (size_t)c->cap_bricks * 8));
  A(dalloc(&c->coarse_inv, 64 * 64));
  A(dalloc(&c->coarse_ok, 1));
  if (rc == MAC_OK) A(check(cudaMemset(c->coarse_ok, 0, sizeof(int))));
  c->npartial = 2 * c->cap_bricks + 64;
  A(dalloc(&c->partial, c->npartial));
  c->mg_float = c->prm.solver == MAC_SOLVER_MGPCG_MIXED || c->prm.solver == MAC_SOLVER_LEARNED_MIXED;
  size_t ts = c->mg_float ? 4 : 8;
  for (int l = 0; l < 3; ++l) {
    size_t n = (size_t)c->cap_bricks * (size_t)((8 >> l) * (8 >> l) * (8 >> l));
    A(check(cudaMalloc(&c->mg_e[l], ts * n)));
    A(check(cudaMalloc(&c->mg_e2[l], ts * n)));
    if (l > 0) {
      A(check(cudaMalloc(&c->mg_r[l], ts * n)));
      A(check(cudaMalloc(&c->mg_w[l], ts * n * 6)));
    }
  }
  if (rc == MAC_OK) rc = mg_configure(c);
  if (rc == MAC_OK) {
    cudaMemset(c->x, 0, 8 * nc);
    cudaMemset(c->fmask, 0, 2 * nc);
  }
  return rc;
}

void free_solver(Ctx* c) {
  cudaFree(c->fmask); cudaFree(c->x); cudaFree(c->b); cudaFree(c->r); cudaFree(c->r2); cudaFree(c->z); cudaFree(c->pd);
  cudaFree(c->q); cudaFree(c->pd2); cudaFree(c->partial); cudaFree(c->dbl); cudaFree(c->dense_buf);
  cudaFree(c->dbl_map); cudaFree(c->dbl_cnt); cudaFree(c->drow);
  cudaFree(c->zold);
  cudaFree(c->coarse_inv);
  cudaFree(c->coarse_ok);
  for (int l = 0; l < kLevels; ++l) {
    cudaFree(c->mg_e[l]); cudaFree(c->mg_e2[l]); cudaFree(c->mg_r[l]); cudaFree(c->mg_w[l]);
  }
}

// ------------------------------------------------------------ helpers
// Sums the per-block partials in a fixed order (one block of 1024 threads).
// Each thread first adds a strided run of partials with eight loads of each
// array in flight (the partials sit in L2; a loop with one load per
// iteration waited one L2 round trip per element).
__device__ inline void sum_partials(const double* partial, int nblk, double* s0, double* s1) {
  __shared__ double sa[32], sb[32];
  double a = 0, b = 0;
  const int step = blockDim.x;
  int i = threadIdx.x;
  for (; i + 7 * step < nblk; i += 8 * step) {
    double va[8], vb[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      va[k] = __ldcg(partial + i + k * step);
      vb[k] = __ldcg(partial + nblk + i + k * step);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      a += va[k];
      b += vb[k];
    }
  }
  for (; i < nblk; i += step) {
    a += __ldcg(partial + i);
    b += __ldcg(partial + nblk + i);
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sa[w] = a;
    sb[w] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0, tb = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
      ta += sa[i];
      tb += sb[i];
    }
    *s0 = ta;
    *s1 = tb;
  }
}

// ------------------------------------------------------- system set-up
// Face classes of every in-domain cell (the assembly loop of
// src/Algorithms_Solve_Pressure.h:103-136): bit f (interior coupling) and bit
// 8+f (face counts in the diagonal); Neumann faces have neither. The Neumann
// test is Data_CellType_Interface_Constant::GetIsConstantInterface_Impl
// (src/Data_CellType_Interface_Constant.h:45-61): only for a valid neighbour;
// sign +1 looks at the neighbour's left face, sign -1 at the cell's own. Bricks
// with an in-domain cell are collected into the domain brick list, and their
// key bounds into the scalars.
__global__ void __launch_bounds__(512) k_fmask(const int* __restrict__ blist, const int* __restrict__ nbr,
                                               const int* __restrict__ bkey, const int8_t* __restrict__ lay,
                                               const uint8_t* __restrict__ type, const uint8_t* __restrict__ flags,
                                               uint16_t* fmask, int* dbl, Scalars* ds) {
  __shared__ int64_t sb[6];
  int b = blist[blockIdx.x];
  load_face_bases(nbr, b, sb);
  __syncthreads();
  int o = threadIdx.x;
  int64_t c = (int64_t)b * kCells + o;
  // every load is issued before any is tested (a missing neighbour brick
  // reads the cell itself)
  const int8_t lc = lay[c];
  const uint8_t tc = type[c], fc = flags[c];
  int64_t nn[6];
  int8_t ln[6];
  uint8_t fn[6], tn[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    nn[f] = nb0(sb, c, o, f);
    const int64_t q = nn[f] < 0 ? c : nn[f];
    ln[f] = lay[q];
    fn[f] = flags[q];
    tn[f] = type[q];
  }
  uint16_t m = 0;
  if (lc != kMissing && is_fluid(tc)) {
    m = kDomainBit;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      int ax = f >> 1;
      if (nn[f] < 0 || ln[f] == kMissing) {
        m |= (uint16_t)(1u << (8 + f));  // missing neighbour: Dirichlet
        continue;
      }
      bool neumann = (f & 1) ? ((fn[f] >> ax) & 1) : ((fc >> ax) & 1);
      if (neumann) continue;
      m |= (uint16_t)(1u << (8 + f));
      if (is_fluid(tn[f])) m |= (uint16_t)(1u << f);
    }
  }
  fmask[c] = m;
  int any = __syncthreads_count(m != 0);
  if (threadIdx.x == 0 && any) {
    atomicAdd((unsigned long long*)&ds->nunknown, (unsigned long long)any);
    dbl[atomicAdd(&ds->ndom, 1)] = b;
    for (int a = 0; a < 3; ++a) {
      atomicMin(&ds->bbox[a], bkey[3 * b + a]);
      atomicMax(&ds->bbox[3 + a], bkey[3 * b + a]);
    }
  }
}

// ------------------------------------------------ canonical domain-brick order
// k_fmask appends the domain bricks in whatever order its blocks finish, and
// the CG adds its per-block partial sums in the order of that list, so without
// a fixed order two runs of the same step differ in the last bits. The list is
// rewritten in the order of the bricks' coordinates (x fastest, then y, z):
// each brick is scattered to its slot in the bounding box (no two share one),
// and the occupied slots are compacted in slot order.
constexpr int kOrderBlock = 1024;
constexpr int64_t kOrderMaxSlots = (int64_t)1 << 26;  // larger boxes keep the appended order

__global__ void k_order_scatter(const int* __restrict__ dbl, int nd, const int* __restrict__ bkey, DenseGrid g,
                                int* __restrict__ map) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nd) return;
  int b = dbl[i];
  map[g.index(bkey[3 * b], bkey[3 * b + 1], bkey[3 * b + 2])] = b;
}

__global__ void __launch_bounds__(kOrderBlock) k_order_count(const int* __restrict__ map, int64_t n,
                                                             int* __restrict__ cnt) {
  int64_t i = (int64_t)blockIdx.x * kOrderBlock + threadIdx.x;
  int k = __syncthreads_count(i < n && map[i] >= 0);
  if (threadIdx.x == 0) cnt[blockIdx.x] = k;
}

// Exclusive prefix sum of nb block counts in place, one block: each thread
// sums a contiguous run, the run totals are scanned through shared memory.
__global__ void __launch_bounds__(kOrderBlock) k_order_scan(int* cnt, int nb) {
  __shared__ int tot[kOrderBlock];
  const int per = (nb + kOrderBlock - 1) / kOrderBlock;
  const int lo = threadIdx.x * per, hi = min(nb, lo + per);
  int s = 0;
  for (int j = lo; j < hi; ++j) s += cnt[j];
  tot[threadIdx.x] = s;
  __syncthreads();
  for (int d = 1; d < kOrderBlock; d <<= 1) {
    int v = threadIdx.x >= d ? tot[threadIdx.x - d] : 0;
    __syncthreads();
    tot[threadIdx.x] += v;
    __syncthreads();
  }
  int run = tot[threadIdx.x] - s;
  for (int j = lo; j < hi; ++j) {
    int v = cnt[j];
    cnt[j] = run;
    run += v;
  }
}

__global__ void __launch_bounds__(kOrderBlock) k_order_write(const int* __restrict__ map, int64_t n,
                                                             const int* __restrict__ off, int* __restrict__ dbl) {
  __shared__ int wsum[kOrderBlock / 32];
  int64_t i = (int64_t)blockIdx.x * kOrderBlock + threadIdx.x;
  int b = i < n ? map[i] : -1;
  unsigned bal = __ballot_sync(0xffffffffu, b >= 0);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) wsum[w] = __popc(bal);
  __syncthreads();
  int before = 0;
  for (int k = 0; k < w; ++k) before += wsum[k];
  if (b >= 0) dbl[off[blockIdx.x] + before + __popc(bal & ((1u << lane) - 1u))] = b;
}

__global__ void k_drow(const int* __restrict__ dbl, int nd, const int* __restrict__ nbr, int* __restrict__ drow) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 8 * (int64_t)nd) return;
  const int k = (int)(t & 7);
  const int b = dbl[t >> 3];
  int v = -1;
  if (k == 0) {
    v = b;
  } else if (k < 7) {
    const int f = k - 1, d = (f & 1) ? 1 : -1, ax = f >> 1;
    v = nbr[(size_t)b * kNbr + nbr_index(ax == 0 ? d : 0, ax == 1 ? d : 0, ax == 2 ? d : 0)];
  }
  drow[t] = v;
}

static int order_domain_bricks(Ctx* c) {
  const int* bb = c->hs->bbox;
  const int nd = c->ndom_host;
  if (nd <= 1) return MAC_OK;
  DenseGrid g;
  g.x0 = bb[0];
  g.y0 = bb[1];
  g.z0 = bb[2];
  g.nx = bb[3] - bb[0] + 1;
  g.ny = bb[4] - bb[1] + 1;
  g.nz = bb[5] - bb[2] + 1;
  const int64_t n = (int64_t)g.nx * g.ny * g.nz;
  if (g.nx < 1 || g.ny < 1 || g.nz < 1 || n > kOrderMaxSlots) return MAC_OK;
  const int64_t nb = (n + kOrderBlock - 1) / kOrderBlock;
  if (n > c->dbl_map_n) {
    cudaFree(c->dbl_map);
    cudaFree(c->dbl_cnt);
    c->dbl_map = nullptr;
    c->dbl_cnt = nullptr;
    c->dbl_map_n = 0;
    int rc = check(cudaMalloc((void**)&c->dbl_map, sizeof(int) * n));
    if (!rc) rc = check(cudaMalloc((void**)&c->dbl_cnt, sizeof(int) * nb));
    if (rc) return rc;
    c->dbl_map_n = n;
  }
  cudaStream_t st = c->stream;
  int rc = check(cudaMemsetAsync(c->dbl_map, 0xff, sizeof(int) * n, st));
  if (rc) return rc;
  k_order_scatter<<<(nd + 255) / 256, 256, 0, st>>>(c->dbl, nd, c->bkey, g, c->dbl_map); MAC_COUNT(c);
  k_order_count<<<(unsigned)nb, kOrderBlock, 0, st>>>(c->dbl_map, n, c->dbl_cnt); MAC_COUNT(c);
  k_order_scan<<<1, kOrderBlock, 0, st>>>(c->dbl_cnt, (int)nb); MAC_COUNT(c);
  k_order_write<<<(unsigned)nb, kOrderBlock, 0, st>>>(c->dbl_map, n, c->dbl_cnt, c->dbl); MAC_COUNT(c);
  return check(cudaGetLastError());
}

__global__ void k_setup_reset(Scalars* ds) {
  ds->nunknown = 0;
  ds->ndom = 0;
  for (int a = 0; a < 3; ++a) {
    ds->bbox[a] = 0x3fffffff;
    ds->bbox[3 + a] = -0x3fffffff;
  }
}

// ------------------------------------------------------------ Dirichlet air
// Policy_Dirichlet_Boundary (src/Policy_Dirichlet_Boundary.h:27-109) over the
// live bricks, for the viscous projection. "Air" there is GetIsAir, which the
// cell-type map answers true for air and for solid cells
// (src/Data_CellType_Fluid_Air_Solid_Inflow.tpp:21-35), i.e. !is_fluid. A
// Dirichlet cell is an existing air cell with an existing non-air face
// neighbour; its pressure is
//   p_D = - sum over such neighbours (i, s) of 2 nu (u_i(c+e_i) - u_i(c)) / h_i * s
// on speed buffer U, in the reference's (i, s) order. pdir gets p_D there and
// NaN everywhere else (every slot of every live brick is written).
__global__ void __launch_bounds__(512) k_dirichlet(const int* __restrict__ blist, const int* __restrict__ nbr,
                                                   const int8_t* __restrict__ lay, const uint8_t* __restrict__ type,
                                                   const double* __restrict__ ux, const double* __restrict__ uy,
                                                   const double* __restrict__ uz, double* __restrict__ pdir,
                                                   Params P) {
  __shared__ int64_t sb[6];
  int b = blist[blockIdx.x];
  load_face_bases(nbr, b, sb);
  __syncthreads();
  int o = threadIdx.x;
  int64_t c = (int64_t)b * kCells + o;
  double out = __longlong_as_double(0x7ff8000000000000ll);
  if (lay[c] != kMissing && !is_fluid(type[c])) {
    const double* U[3] = {ux, uy, uz};
    double ret = 0;
    bool db = false;
    for (int i = 0; i < 3; ++i) {
      for (int s = -1; s <= 1; s += 2) {
        int64_t n = nb0(sb, c, o, 2 * i + (s > 0));
        if (n >= 0 && lay[n] != kMissing && is_fluid(type[n])) {
          db = true;
          const double v1 = U[i][c];
          const int64_t n2 = nb0(sb, c, o, 2 * i + 1);
          const double v2 = n2 < 0 ? 0.0 : U[i][n2];
          ret -= 2 * P.nu * (v2 - v1) * P.ih[i] * s;
        }
      }
    }
    if (db) out = ret;
  }
  pdir[c] = out;
}

// ------------------------------------------------------------ CG kernels
// Divergence (Policy_Divergence::Get_Divergence, src/Policy_Divergence.h:20-29)
// of speed buffer ib into rhs = -div (the right-hand side of M x = -div) and
// the block's partial |div|^2; x starts at 0 or, warm, at the cell pressure.
// With Dirichlet air pressures (pdir non-null, the viscous projection of
// src/Algorithms_Solve_Pressure_Dirichlet.h:178-188), a cell next to a
// Dirichlet cell first takes div -= sum over those neighbours of p_D / h_i^2.
__global__ void __launch_bounds__(kBT) k_divergence(const int* __restrict__ drow,
                                                    const uint16_t* __restrict__ fmask, const double* __restrict__ ux,
                                                    const double* __restrict__ uy, const double* __restrict__ uz,
                                                    const double* __restrict__ pres, double* __restrict__ rhs,
                                                    double* __restrict__ x, double* __restrict__ r, int warm,
                                                    double* partial, Params P, const double* __restrict__ pdir) {
  __shared__ int64_t sb[6];
  const int b = load_drow(drow, sb);
  __syncthreads();
  double bb = 0;
#pragma unroll
  for (int k = 0; k < kCPT; ++k) {
    int o = threadIdx.x + kBT * k;
    int64_t c = (int64_t)b * kCells + o;
    // the mask and all six speeds are loaded before either is tested (a
    // missing neighbour brick reads the cell itself)
    const uint16_t m = fmask[c];
    const double* U[3] = {ux, uy, uz};
    int64_t nn[3];
    double uc[3], un[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      nn[i] = nb0(sb, c, o, 2 * i + 1);
      uc[i] = U[i][c];
      un[i] = U[i][nn[i] < 0 ? c : nn[i]];
    }
    if (!(m & kDomainBit)) {
      rhs[c] = 0.0;
      x[c] = 0.0;
      r[c] = 0.0;
      continue;
    }
    double d = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      d -= uc[i] * P.ih[i];
      d += (nn[i] < 0 ? 0.0 : un[i]) * P.ih[i];
    }
    if (pdir) {
      double sum = 0;
      bool any = false;
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        int64_t n = nb0(sb, c, o, f);
        double q = n < 0 ? 0.0 : pdir[n];
        if (n >= 0 && q == q) {
          any = true;
          sum += q * P.ih[f >> 1] * P.ih[f >> 1];
        }
      }
      if (any) d -= sum;
    }
    rhs[c] = -d;
    r[c] = -d;
    x[c] = warm ? pres[c] : 0.0;
    bb += d * d;
  }
  block_sum<kBT>(bb, 0.0, partial);
}

__device__ inline double apply0(const double* __restrict__ v, const uint16_t* __restrict__ fmask, const int64_t* sb,
                                int64_t c, int o, uint16_t m, const Params& P) {
  double vc = v[c];
  double s = 0;
  for (int f = 0; f < 6; ++f) {
    if (m & (1u << (8 + f))) s += P.ih2[f >> 1] * vc;
    if (m & (1u << f)) s -= P.ih2[f >> 1] * v[nb0(sb, c, o, f)];
  }
  return s;
}

// r = rhs - M x for a warm start, with the block's partial r.r
__global__ void __launch_bounds__(kBT) k_residual(const int* __restrict__ drow,
                                                  const uint16_t* __restrict__ fmask, const double* __restrict__ rhs,
                                                  const double* __restrict__ x, double* __restrict__ r,
                                                  double* partial, Params P) {
  __shared__ int64_t sb[6];
  const int b = load_drow(drow, sb);
  __syncthreads();
  double rr = 0;
#pragma unroll
  for (int k = 0; k < kCPT; ++k) {
    int o = threadIdx.x + kBT * k;
    int64_t c = (int64_t)b * kCells + o;
    uint16_t m = fmask[c];
    if (m & kDomainBit) {
      double v = rhs[c] - apply0(x, fmask, sb, c, o, m, P);
      r[c] = v;
      rr += v * v;
    }
  }
  block_sum<kBT>(rr, 0.0, partial);
}

// p = z + beta p (first: p = z), then q = M p and the partial p.q; the
// neighbours' new p is formed on the fly so p is read once and written once.
__global__ void __launch_bounds__(kBT) k_update_spmv(const int* __restrict__ drow,
                                                     const uint16_t* __restrict__ fmask, const double* __restrict__ z,
                                                     const double* __restrict__ pold, double* __restrict__ pnew,
                                                     double* __restrict__ q, double* partial, Params P,
                                                     const Scalars* ds, int first) {
  __shared__ int64_t sb[6];
  __shared__ double sp[kS1];  // the new direction on the brick and its face halo
  // prologue: brick, face neighbours and face masks (static), the brick's z
  // (the preconditioner's output, two launches back) and p_old (16-byte
  // vector loads); only beta comes from the previous launch
  const int b = load_drow(drow, sb);
  const int ob = zrun_base();  // the stencil pass's z-run (cells ob + 64 k)
  uint16_t mk[kCPT];
#pragma unroll
  for (int k = 0; k < kCPT; ++k) mk[k] = fmask[(int64_t)b * kCells + ob + 64 * k];
  const int o4 = 4 * threadIdx.x;
  double vz[4], vp[4] = {0.0, 0.0, 0.0, 0.0};
  load4(z + (int64_t)b * kCells + o4, vz);
  if (!first) load4(pold + (int64_t)b * kCells + o4, vp);
  pdl_entry();
  if (ds->done) return;
  const double be = first ? 0.0 : ds->beta;
  __syncthreads();
  // p = z (first) or z + beta p_old, on the brick and its face halo
  if (first) stage_h1_halo(sp, sb, [&](int64_t i) { return z[i]; });
  else stage_h1_halo(sp, sb, [&](int64_t i) { return z[i] + be * pold[i]; });
  const int si4 = s1_of(o4);
#pragma unroll
  for (int k = 0; k < 4; ++k) sp[si4 + k] = first ? vz[k] : vz[k] + be * vp[k];
  __syncthreads();
  const int si0 = s1_of(ob);
  double pcs[kCPT];
#pragma unroll
  for (int k = 0; k < kCPT; ++k) pcs[k] = sp[si0 + 100 * k];
  double pq = 0;
#pragma unroll
  for (int k = 0; k < kCPT; ++k) {
    const int64_t c = (int64_t)b * kCells + ob + 64 * k;
    const uint16_t m = mk[k];
    if (!(m & kDomainBit)) {
      pnew[c] = 0.0;
      q[c] = 0.0;
      continue;
    }
    const int si = si0 + 100 * k;
    const double pc = pcs[k];
    double s = 0;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      if (m & (1u << (8 + f))) s += P.ih2[f >> 1] * pc;
      if (m & (1u << f)) s -= P.ih2[f >> 1] * zrun_nbr(sp, pcs, si, k, f);
    }
    pnew[c] = pc;
    q[c] = s;
    pq += pc * s;
  }
  block_sum<kBT>(pq, 0.0, partial);
}

__global__ void k_fin_alpha(const double* partial, int nblk, Scalars* ds) {
  pdl_entry();
  if (ds->done) return;
  double pq, unused;
  sum_partials(partial, nblk, &pq, &unused);
  if (threadIdx.x == 0) {
    ds->pq = pq;
    ds->alpha = pq != 0 ? ds->rz / pq : 0.0;
  }
}

// x += alpha p, r -= alpha q, partial r.r
__global__ void __launch_bounds__(512) k_axpy(const int* __restrict__ dbl, double* __restrict__ x,
                                              double* __restrict__ r, const double* __restrict__ p,
                                              const double* __restrict__ q, double* partial, const Scalars* ds) {
  pdl_entry();
  if (ds->done) return;
  double a = ds->alpha;
  int64_t c = (int64_t)dbl[blockIdx.x] * kCells + threadIdx.x;
  x[c] += a * p[c];
  double rv = r[c] - a * q[c];
  r[c] = rv;
  block_sum<512>(rv * rv, 0.0, partial);
}

__global__ void k_fin_rr(const double* partial, int nblk, Scalars* ds, double rtol2, int max_iters) {
  pdl_entry();
  if (ds->done) return;
  double rr, unused;
  sum_partials(partial, nblk, &rr, &unused);
  if (threadIdx.x == 0) {
    ds->rr = rr;
    ds->iters += 1;
    if (rr <= rtol2 * ds->bnorm2 || ds->iters >= max_iters || !(rr == rr)) ds->done = 1;
  }
}

__global__ void k_fin_bnorm(const double* partial, int nblk, Scalars* ds) {
  double bb, unused;
  sum_partials(partial, nblk, &bb, &unused);
  if (threadIdx.x == 0) {
    ds->bnorm2 = bb;
    ds->rr = bb;
    ds->iters = 0;
    ds->done = bb == 0 ? 1 : 0;
  }
}

__global__ void k_fin_rr_initial(const double* partial, int nblk, Scalars* ds, double rtol2) {
  double rr, unused;
  sum_partials(partial, nblk, &rr, &unused);
  if (threadIdx.x == 0) {
    ds->rr = rr;
    if (rr <= rtol2 * ds->bnorm2) ds->done = 1;
  }
}

// beta = rz_new / rz
__global__ void k_fin_beta(const double* partial, int nblk, Scalars* ds, int first) {
  pdl_entry();
  if (ds->done) return;
  double rz, unused;
  sum_partials(partial, nblk, &rz, &unused);
  if (threadIdx.x == 0) {
    ds->beta = first ? 0.0 : (ds->rz != 0 ? rz / ds->rz : 0.0);
    ds->rz = rz;
  }
}

// Jacobi preconditioner (MAC_SOLVER_CG_FP64): z = r / diag, with the r.z partials.
__global__ void __launch_bounds__(512) k_jacobi_prec(const int* __restrict__ dbl, const uint16_t* __restrict__ fmask,
                                                     const double* __restrict__ r, double* __restrict__ z,
                                                     double* partial, Params P) {
  pdl_entry();
  int64_t c = (int64_t)dbl[blockIdx.x] * kCells + threadIdx.x;
  uint16_t m = fmask[c];
  double v = (m & kDomainBit) ? r[c] * P.dtab[active_index(m)] : 0.0;
  z[c] = v;
  block_sum<512>(r[c] * v, 0.0, partial);
}

// Pressure write-back and velocity correction, fused
// (src/Algorithms_Solve_Pressure.h:185-207): existing cells get p = x in the
// domain, p_D on Dirichlet air cells of the viscous projection
// (src/Algorithms_Solve_Pressure_Dirichlet.h:196-208) and 0 elsewhere; face i of a cell in the domain, or whose -e_i
// neighbour is, gets u_i -= p(c)/h_i - p(c-e_i)/h_i
// (Policy_Gradiant::Get_Gradiant, src/Policy_Gradiant.h:32-37) through the
// non-forced Set (const faces keep their value).
__device__ inline double dir_or_zero(double q) { return q == q ? q : 0.0; }

__global__ void __launch_bounds__(512) k_gradient(const int* __restrict__ blist, const int* __restrict__ nbr,
                                                  const int8_t* __restrict__ lay, const uint8_t* __restrict__ type,
                                                  const uint8_t* __restrict__ flags, const double* __restrict__ x,
                                                  double* __restrict__ pres, double* ux, double* uy, double* uz,
                                                  Params P, const double* __restrict__ pdir) {
  __shared__ int64_t sb[6];
  int b = blist[blockIdx.x];
  load_face_bases(nbr, b, sb);
  __syncthreads();
  int o = threadIdx.x;
  int64_t c = (int64_t)b * kCells + o;
  // every load a cell may need is issued before any is tested (a missing
  // neighbour brick reads the cell itself), so no load waits on another
  int64_t nn[3];
  int8_t ln[3];
  uint8_t tn[3];
  double xn[3];
  double* U[3] = {ux, uy, uz};
  const int8_t lc = lay[c];
  const uint8_t tc = type[c], fl = flags[c];
  const double xc = x[c];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    nn[i] = nb0(sb, c, o, 2 * i);
    const int64_t m = nn[i] >= 0 ? nn[i] : c;
    ln[i] = lay[m];
    tn[i] = type[m];
    xn[i] = x[m];
  }
  if (lc == kMissing) return;
  const bool dc = is_fluid(tc);
  const double pc = dc ? xc : (pdir ? dir_or_zero(pdir[c]) : 0.0);
  pres[c] = pc;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const int64_t n = nn[i];
    const bool nexists = n >= 0 && ln[i] != kMissing;
    const bool dn = nexists && is_fluid(tn[i]);
    if (!(dc || dn)) continue;
    if (fl & (1u << i)) continue;
    const double pn = nexists ? (dn ? xn[i] : (pdir ? dir_or_zero(pdir[n]) : 0.0)) : (n >= 0 ? pres[n] : 0.0);
    double gr = pc * P.ih[i];
    gr -= pn * P.ih[i];
    U[i][c] = U[i][c] - gr;
  }
}

// max |div| over domain cells (the check of src/Algorithms_Solve_Pressure.h:208-219)
__global__ void __launch_bounds__(kBT) k_divmax(const int* __restrict__ drow,
                                                const uint16_t* __restrict__ fmask, const double* __restrict__ ux,
                                                const double* __restrict__ uy, const double* __restrict__ uz, Params P,
                                                Scalars* ds) {
  __shared__ int64_t sb[6];
  const int b = load_drow(drow, sb);
  __syncthreads();
  double mx = 0;
#pragma unroll
  for (int k = 0; k < kCPT; ++k) {
    int o = threadIdx.x + kBT * k;
    int64_t c = (int64_t)b * kCells + o;
    const uint16_t m = fmask[c];
    const double* U[3] = {ux, uy, uz};
    int64_t nn[3];
    double uc[3], un[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      nn[i] = nb0(sb, c, o, 2 * i + 1);
      uc[i] = U[i][c];
      un[i] = U[i][nn[i] < 0 ? c : nn[i]];
    }
    if (!(m & kDomainBit)) continue;
    double d = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      d -= uc[i] * P.ih[i];
      d += (nn[i] < 0 ? 0.0 : un[i]) * P.ih[i];
    }
    mx = fmax(mx, fabs(d));
  }
  for (int s = 16; s > 0; s >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, s));
  if ((threadIdx.x & 31) == 0) atomicMax(&ds->div_bits, (unsigned long long)__double_as_longlong(mx));
}

__global__ void k_zero_div(Scalars* ds) { ds->div_bits = 0; }

// ------------------------------------------------------------ drivers
// ------------------------------------------- learned preconditioner glue
// The domain's bounding box of bricks as a dense grid (x fastest): residual
// (FP32) and the network's cell mask (1 in the domain, -1 solid, 0 otherwise:
// air and missing cells are Dirichlet), one block per brick of the box.
__global__ void __launch_bounds__(512) k_to_dense(const unsigned long long* __restrict__ hk,
                                                  const int* __restrict__ hv, int64_t hcap,
                                                  const int8_t* __restrict__ lay, const uint8_t* __restrict__ type,
                                                  const uint16_t* __restrict__ fmask, const double* __restrict__ r,
                                                  int bx, int by, int bz, int nbx, int nby, float* rd, int8_t* md) {
  const int i = blockIdx.x;
  const int kx = i % nbx, ky = (i / nbx) % nby, kz = i / (nbx * nby);
  __shared__ int b;
  if (threadIdx.x == 0) b = hash_find(hk, hv, hcap, pack_key(bx + kx, by + ky, bz + kz));
  __syncthreads();
  const int o = threadIdx.x;
  const int x = kx * 8 + (o & 7), y = ky * 8 + ((o >> 3) & 7), z = kz * 8 + (o >> 6);
  const size_t di = ((size_t)z * (nby * 8) + y) * (size_t)(nbx * 8) + x;
  float rv = 0.0f;
  int8_t mv = 0;
  if (b >= 0) {
    const int64_t c = (int64_t)b * kCells + o;
    if (fmask[c] & kDomainBit) {
      rv = (float)r[c];
      mv = 1;
    } else if (lay[c] != kMissing && type[c] == MAC_CELL_SOLID) {
      mv = -1;
    }
  }
  rd[di] = rv;
  md[di] = mv;
}

// z = scale * (network correction) on domain cells, 0 elsewhere, then one
// weighted Jacobi step z += omega D^-1 (r - M z) (omega = 0: none; the
// neighbours' corrections are read from the dense grid); partials of r.z (new)
// and r.zold for the flexible (Polak-Ribiere) beta.
__global__ void __launch_bounds__(512) k_from_dense(const int* __restrict__ dbl, const int* __restrict__ bkey,
                                                    const uint16_t* __restrict__ fmask, const float* __restrict__ zd,
                                                    int bx, int by, int bz, int nbx, int nby, double scale,
                                                    double omega, const double* __restrict__ r,
                                                    const double* __restrict__ zold, double* __restrict__ z,
                                                    double* partial, Params P) {
  const int b = dbl[blockIdx.x];
  const int o = threadIdx.x;
  const int64_t c = (int64_t)b * kCells + o;
  const int x = (bkey[3 * b] - bx) * 8 + (o & 7), y = (bkey[3 * b + 1] - by) * 8 + ((o >> 3) & 7),
            zz = (bkey[3 * b + 2] - bz) * 8 + (o >> 6);
  const uint16_t m = fmask[c];
  double v = 0.0, rz = 0.0, rzo = 0.0;
  if (m & kDomainBit) {
    const int64_t sx = 1, sy = (int64_t)nbx * 8, sz = sy * (int64_t)(nby * 8);
    const int64_t di = zz * sz + y * sy + x;
    v = scale * (double)zd[di];
    if (omega > 0.0) {
      const int64_t off[6] = {-sx, sx, -sy, sy, -sz, sz};
      double mz = 0.0;
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        if (m & (1u << (8 + f))) mz += P.ih2[f >> 1] * v;
        if (m & (1u << f)) mz -= P.ih2[f >> 1] * scale * (double)zd[di + off[f]];
      }
      v += omega * P.dtab[active_index(m)] * (r[c] - mz);
    }
    rz = r[c] * v;
    rzo = r[c] * zold[c];
  }
  z[c] = v;
  block_sum<512>(rz, rzo, partial);
}

// beta = (r.z - r.zold) / rz_prev (Polak-Ribiere; 0 on a restart), rz = r.z
__global__ void k_fin_beta_flex(const double* partial, int nblk, Scalars* ds, int first) {
  if (ds->done) return;
  double rz, rzo;
  sum_partials(partial, nblk, &rz, &rzo);
  if (threadIdx.x == 0) {
    ds->beta = first ? 0.0 : (ds->rz != 0 ? (rz - rzo) / ds->rz : 0.0);
    ds->rz = rz;
  }
}

bool learned_solver(const Ctx* c) {
  return (c->prm.solver == MAC_SOLVER_LEARNED || c->prm.solver == MAC_SOLVER_LEARNED_MIXED) && c->unet;
}

// Allocates (once) and clears the previous-z vector of the flexible CG.
int learned_begin(Ctx* c) {
  if (!c->zold) {
    int rc = check(cudaMalloc((void**)&c->zold, 8 * (size_t)c->cap_bricks * kCells));
    if (rc) return rc;
  }
  return check(cudaMemsetAsync(c->zold, 0, 8 * (size_t)c->cap_bricks * kCells, c->stream));
}

// z = network(r) on the domain's brick box (+ the Jacobi step), then beta.
int learned_precondition(Ctx* c, int first) {
  const int* bb = c->hs->bbox;
  const int nbx = bb[3] - bb[0] + 1, nby = bb[4] - bb[1] + 1, nbz = bb[5] - bb[2] + 1;
  float *rd = nullptr, *zd = nullptr;
  int8_t* md = nullptr;
  int rc = unet::stage((unet::Net*)c->unet, 1, nbz * 8, nby * 8, nbx * 8, &rd, &md, &zd);
  if (rc) return rc;
  cudaStream_t st = c->stream;
  std::swap(c->z, c->zold);
  k_to_dense<<<nbx * nby * nbz, 512, 0, st>>>(c->hkeys, c->hval, c->hcap, c->lay, c->type, c->fmask, c->r, bb[0],
                                              bb[1], bb[2], nbx, nby, rd, md); MAC_COUNT(c);
  rc = unet::apply((unet::Net*)c->unet, st);
  if (rc) return rc;
  // the network inverts the unit-spacing operator; M = (unit operator) / h^2
  const double scale = 1.0 / c->dp.ih2[0];
  k_from_dense<<<c->ndom_host, 512, 0, st>>>(c->dbl, c->bkey, c->fmask, zd, bb[0], bb[1], bb[2], nbx, nby, scale,
                                             c->learned_omega, c->r, c->zold, c->z, c->partial, c->dp); MAC_COUNT(c);
  k_fin_beta_flex<<<1, 1024, 0, st>>>(c->partial, c->ndom_host, c->ds, first); MAC_COUNT(c);
  return check(cudaGetLastError());
}

int setup_system(Ctx* c) {
  cudaStream_t st = c->stream;
  int n = c->nlive_host;
  prof_begin(c, PH_SETUP);
  k_setup_reset<<<1, 1, 0, st>>>(c->ds); MAC_COUNT(c);
  if (n > 0) {
    k_fmask<<<n, 512, 0, st>>>(c->blist, c->nbr, c->bkey, c->lay, c->type, c->flags, c->fmask, c->dbl, c->ds); MAC_COUNT(c);
  }
  int rc = read_scalars(c);
  if (rc) return rc;
  c->ndom_host = c->hs->ndom;
  c->stats.unknowns = c->hs->nunknown;
  if ((rc = order_domain_bricks(c))) return rc;
  if (c->ndom_host > 0) {
    k_drow<<<grid_for(8 * (int64_t)c->ndom_host, 256), 256, 0, st>>>(c->dbl, c->ndom_host, c->nbr, c->drow); MAC_COUNT(c);
  }
  if (c->ndom_host > 0 && c->prm.solver != MAC_SOLVER_CG_FP64) {
    rc = mg_setup(c);
    if (rc) return rc;
  }
  prof_end(c, PH_SETUP);
  c->system_ready = true;
  return check(cudaGetLastError());
}

static void precondition(Ctx* c) {
  if (c->prm.solver == MAC_SOLVER_CG_FP64) {
    launch_k(c, k_jacobi_prec, c->ndom_host, 512, 0, c->dbl, c->fmask, c->r, c->z, c->partial, c->dp); MAC_COUNT(c);
  } else {
    mg_vcycle(c, 0, 3);
  }
}

// Convergence test after the update the V-cycle's first kernel applied (its
// partial r.r are in c->partial).
void cg_finish_update(Ctx* c) {
  launch_k(c, k_fin_rr, 1, 1024, 0, c->partial, c->npart_head, c->ds, c->prm.rtol * c->prm.rtol,
           c->prm.max_iters); MAC_COUNT(c);
}

int project(Ctx* c, int ib) {
  size_t cap = (size_t)c->cap_bricks * kCells;
  double* U[3] = {c->f64 + (size_t)(3 * ib) * cap, c->f64 + (size_t)(3 * ib + 1) * cap,
                  c->f64 + (size_t)(3 * ib + 2) * cap};
  return project_field(c, U, U);
}

// The projection of vector field U (Divergence_Projection: divergence,
// solve, pressure write-back, gradient correction of U). D is the speed
// field the Dirichlet air pressures of the viscous composition read
// (Speed_GetRef(-1, false), src/Policy_Dirichlet_Boundary.h:100-102): U
// itself, except in the force projection of pipeline B
// (src/Algorithms_Solve_Pressure_Force.h:16-24), where U is the acceleration.
int project_field(Ctx* c, double* const* U, const double* const* D) {
  if (!c->system_ready) {
    int rc = setup_system(c);
    if (rc) return rc;
  }
  int nd = c->ndom_host;
  cudaStream_t st = c->stream;
  size_t cap = (size_t)c->cap_bricks * kCells;
  int status = MAC_OK;
  int rc;
  // the viscous composition projects with Dirichlet air pressures
  double* pdir = c->dp.nu > 0 ? c->pdir : nullptr;
  if (pdir && nd == 0 && c->nlive_host > 0) {
    k_dirichlet<<<c->nlive_host, 512, 0, st>>>(c->blist, c->nbr, c->lay, c->type, D[0], D[1], D[2], pdir,
                                               c->dp); MAC_COUNT(c);
  }
  if (nd > 0) {
    int warm = c->prm.warm_start ? 1 : 0;
    double rtol2 = c->prm.rtol * c->prm.rtol;
    prof_begin(c, PH_DIVERGENCE);
    if (pdir) {
      k_dirichlet<<<c->nlive_host, 512, 0, st>>>(c->blist, c->nbr, c->lay, c->type, D[0], D[1], D[2], pdir,
                                                 c->dp); MAC_COUNT(c);
    }
    k_divergence<<<nd, kBT, 0, st>>>(c->drow, c->fmask, U[0], U[1], U[2], c->f64 + (size_t)PRES * cap, c->b,
                                     c->x, c->r, warm, c->partial, c->dp, pdir); MAC_COUNT(c);
    prof_end(c, PH_DIVERGENCE);
    k_fin_bnorm<<<1, 1024, 0, st>>>(c->partial, nd, c->ds); MAC_COUNT(c);
    if (warm) {
      k_residual<<<nd, kBT, 0, st>>>(c->drow, c->fmask, c->b, c->x, c->r, c->partial, c->dp); MAC_COUNT(c);
      k_fin_rr_initial<<<1, 1024, 0, st>>>(c->partial, nd, c->ds, rtol2); MAC_COUNT(c);
    }
    // a step's particle binning runs beside this solve's iterations
    if ((rc = launch_side_binning(c))) return rc;
    int first = 1;
    // Learned preconditioner: flexible CG until it stalls (the residual norm
    // falls by less than 2x over kStallWindow iterations, or kLearnedMax
    // iterations pass), then MG-PCG restarts from the current iterate.
    bool learned = learned_solver(c);
    if (learned && (rc = learned_begin(c))) return rc;
    constexpr int kStallWindow = 8, kLearnedMax = 200;
    std::vector<double> hist;
    c->stats.learned_iterations = 0;
    // The multigrid forms fold x += alpha p, r -= alpha q and the convergence
    // test into the next V-cycle's first kernel. The host reads each
    // iteration's scalars one iteration late, with the next iteration already
    // enqueued, so the device does not wait for the host between iterations.
    // Once the residual's contraction predicts convergence within two
    // iterations ("near"), the host instead tests right after each V-cycle's
    // first kernel and enqueues the rest only if the solve goes on, so no
    // V-cycle runs past convergence (its kernels would return at once, but
    // some twenty empty launches still cost about 0.1 ms).
    const bool mg = c->prm.solver != MAC_SOLVER_CG_FP64;
    bool lagged = false;  // the fold was used: the final scalars are read at the end
    bool near = false;
    int ahead = 0;        // readbacks enqueued while not near
    double rr_prev = -1;  // r.r of the iteration before the last one read back
    while (true) {
      const bool fold = mg && !learned;
      prof_begin(c, PH_VCYCLE);
      if (learned) {
        if ((rc = learned_precondition(c, first))) return rc;
      } else if (fold) {
        lagged = true;
        const int update = first ? 0 : 1;
        mg_vcycle(c, update, 1);
        if (near && update) {
          rc = read_scalars(c);
          if (rc || c->hs->done) {
            prof_end(c, PH_VCYCLE);
            if (rc) return rc;
            break;
          }
        }
        mg_vcycle(c, 0, 2);
      } else {
        precondition(c);
      }
      prof_end(c, PH_VCYCLE);
      prof_begin(c, PH_CGVEC);
      if (!learned) {
        launch_k(c, k_fin_beta, 1, 1024, 0, c->partial, nd, c->ds, first); MAC_COUNT(c);
      }
      prof_end(c, PH_CGVEC);
      prof_begin(c, PH_SPMV);
      std::swap(c->pd, c->pd2);  // pd2: previous direction, pd: new one
      launch_k(c, k_update_spmv, nd, kBT, 0, c->drow, c->fmask, c->z, c->pd2, c->pd, c->q, c->partial, c->dp, c->ds,
               first); MAC_COUNT(c);
      prof_end(c, PH_SPMV);
      first = 0;
      prof_begin(c, PH_CGVEC);
      launch_k(c, k_fin_alpha, 1, 1024, 0, c->partial, nd, c->ds); MAC_COUNT(c);
      if (!fold) {
        launch_k(c, k_axpy, nd, 512, 0, c->dbl, c->x, c->r, c->pd, c->q, c->partial, c->ds); MAC_COUNT(c);
        launch_k(c, k_fin_rr, 1, 1024, 0, c->partial, nd, c->ds, rtol2, c->prm.max_iters); MAC_COUNT(c);
      }
      prof_end(c, PH_CGVEC);
      if (fold) {
        if (near) continue;  // tested after the next V-cycle's first kernel
        const int s = ahead & 1;
        rc = check(cudaMemcpyAsync(&c->hs_lag[s], c->ds, sizeof(Scalars), cudaMemcpyDeviceToHost, st));
        if (!rc) rc = check(cudaEventRecord(c->ev_lag[s], st));
        if (rc) return rc;
        if (ahead++ == 0) continue;
        if ((rc = check(cudaEventSynchronize(c->ev_lag[s ^ 1])))) return rc;
        const Scalars& h = c->hs_lag[s ^ 1];
        if (h.done) break;
        // r.r two tests after the one read back, at the last contraction
        if (rr_prev > 0) {
          const double q = h.rr / rr_prev;
          near = h.rr * q * q <= 4.0 * rtol2 * h.bnorm2;
        }
        if (h.iters + 2 >= c->prm.max_iters) near = true;
        rr_prev = h.rr;
        continue;
      }
      rc = read_scalars(c);
      if (rc) return rc;
      if (learned) c->stats.learned_iterations = c->hs->iters;
      if (c->hs->done) break;
      if (learned) {
        hist.push_back(c->hs->rr);
        const int k = (int)hist.size();
        const bool stalled = k >= kStallWindow && hist[k - 1] > 0.25 * hist[k - kStallWindow];
        if (stalled || k >= kLearnedMax) {
          // MG-PCG from the current x: true residual, fresh directions
          learned = false;
          c->stats.fallbacks += 1;
          k_residual<<<nd, kBT, 0, st>>>(c->drow, c->fmask, c->b, c->x, c->r, c->partial, c->dp); MAC_COUNT(c);
          k_fin_rr_initial<<<1, 1024, 0, st>>>(c->partial, nd, c->ds, rtol2); MAC_COUNT(c);
          first = 1;
        }
      }
    }
    if (lagged && (rc = read_scalars(c))) return rc;
    double relres = c->hs->bnorm2 > 0 ? sqrt(c->hs->rr / c->hs->bnorm2) : 0.0;
    c->stats.iterations = c->hs->iters;
    c->stats.total_iterations += c->hs->iters;
    c->stats.relres = relres;
    c->stats.solves += 1;
    if (!(relres <= c->prm.rtol)) status = MAC_ERR_NOT_CONVERGED;
  } else {
    c->stats.iterations = 0;
    c->stats.relres = 0.0;
    c->stats.solves += 1;
  }
  int n = c->nlive_host;
  if (n > 0) {
    prof_begin(c, PH_GRADIENT);
    k_gradient<<<n, 512, 0, st>>>(c->blist, c->nbr, c->lay, c->type, c->flags, c->x, c->f64 + (size_t)PRES * cap,
                                  U[0], U[1], U[2], c->dp, pdir); MAC_COUNT(c);
    prof_end(c, PH_GRADIENT);
  }
  if (c->prm.div_check && nd > 0) {
    k_zero_div<<<1, 1, 0, st>>>(c->ds); MAC_COUNT(c);
    k_divmax<<<nd, kBT, 0, st>>>(c->drow, c->fmask, U[0], U[1], U[2], c->dp, c->ds); MAC_COUNT(c);
    rc = read_scalars(c);
    if (rc) return rc;
    unsigned long long bits = c->hs->div_bits;
    std::memcpy(&c->stats.max_div, &bits, sizeof(double));
  }
  rc = check(cudaGetLastError());
  return rc ? rc : status;
}

}  // namespace mac
