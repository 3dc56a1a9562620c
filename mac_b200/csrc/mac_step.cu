// Step orchestration and the stage entry points of the C-ABI, plus the
// drop-in CSC linear solver (the Policy_Solve_Linear_* member functions).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "mac_internal.cuh"

namespace mac {

int rk_stage(Ctx* c, int stage);

// Algorithms_RungeKutta_RK2_TVD::Do (src/Algorithms_RungeKutta_RK2_TVD.h:20-66):
// Init_Iteration (system set-up) once, stage 1 into speed 1, projection of
// speed 1, stage 2 back into speed 0, projection of speed 0.
int rk2tvd(Ctx* c) {
  int rc = setup_system(c);
  if (rc) return rc;
  if ((rc = rk_stage(c, 1))) return rc;
  int s1 = project(c, 1);
  if (s1 && s1 != MAC_ERR_NOT_CONVERGED) return s1;
  if ((rc = rk_stage(c, 2))) return rc;
  int s2 = project(c, 0);
  if (s2) return s2;
  return s1;
}

__global__ void k_advance_time(Scalars* ds) { ds->t += ds->dt; }

// Algorithms_RungeKutta_all::Do (src/Algorithms_RungeKutta_all.h:35-156) with
// the policy of test/Jet3.cpp:642-675: the acceleration is zeroed, then each
// of the four stages runs the stage topology at the current particle position
// (init2), Algorithms_Extrapolate on the stage speed, gravity + convection (+
// viscosity) into the acceleration, the force projection of the acceleration
// (Dirichlet pressures from the stage speed), Algorithms_Extrapolate on the
// acceleration, and the stage's grid and particle updates. The stage speed is
// buffer 0 in stage 1 and buffer 2 after it; the topology reads position 0 in
// stage 1 and position 2 after it.
int rk_all(Ctx* c) {
  if (c->dp.pipeline != 1) return MAC_ERR_INVALID;
  size_t cap = (size_t)c->cap_bricks * kCells;
  double* U0[3] = {c->f64 + U0X * cap, c->f64 + U0Y * cap, c->f64 + U0Z * cap};
  double* U2[3] = {c->u2, c->u2 + cap, c->u2 + 2 * cap};
  double* A[3] = {c->f64 + AX * cap, c->f64 + AY * cap, c->f64 + AZ * cap};
  int rc, status = MAC_OK;
  c->imove = 0;
  if ((rc = acc_zero(c))) return rc;
  for (int stage = 1; stage <= 4; ++stage) {
    double* const* S = stage == 1 ? U0 : U2;
    if ((rc = topology_stage(c))) return rc;
    if ((rc = extrapolate_field(c, S))) return rc;
    if ((rc = forces_add(c, S))) return rc;
    int sp = project_field(c, A, S);
    if (sp && sp != MAC_ERR_NOT_CONVERGED) return sp;
    if (sp) status = sp;
    if ((rc = extrapolate_field(c, A))) return rc;
    if ((rc = rk_all_stage_update(c, stage, S))) return rc;
    if (stage == 1) c->imove = 2;
  }
  c->imove = 0;
  return status;
}

// One step of test/Jet3.cpp:720-726 (pipeline B): the per-step init (the depth
// topology with dt, then Algorithms_Extrapolate) and Algorithms_RungeKutta_all,
// which moves the particles itself.
static int step_b(Ctx* c) {
  int rc = topology_rebuild(c, false);
  if (rc) return rc;
  if ((rc = extrapolate(c))) return rc;
  return rk_all(c);
}

// One step of test/TestJetDEau_Basic.cpp:434-441. The particles do not move
// between the topology and the move, so their binning by brick and cell runs
// on a second stream, started when the first projection's CG loop begins
// (its iterations are latency-bound and leave memory bandwidth free) and
// overlapping the rest of RK2-TVD and the extrapolation; the context's stream
// waits for it before the move, and on every early return, since the binning
// swaps the current particle buffers.
static int step(Ctx* c) {
  if (c->dp.pipeline == 1) return step_b(c);
  int rc = topology_rebuild(c, false);
  if (rc) return rc;
  c->bin_pending = c->bin_side && c->np_host > 0 && c->nlive_host > 0 ? 1 : 0;
  c->bin_launched = 0;
  auto join = [&]() -> int {
    c->bin_pending = 0;
    if (!c->bin_launched) return MAC_OK;
    c->bin_launched = 0;
    return check(cudaStreamWaitEvent(c->stream, c->ev_bins, 0));
  };
  int ode = rk2tvd(c);
  if (ode && ode != MAC_ERR_NOT_CONVERGED) {
    join();
    return ode;
  }
  if ((rc = extrapolate(c))) {
    join();
    return rc;
  }
  const bool binned = c->bin_launched != 0;
  if ((rc = join())) return rc;
  if (binned) {
    prof_begin(c, PH_MOVE);
    rc = move_binned(c);
    prof_end(c, PH_MOVE);
  } else {
    rc = move_particles(c);
  }
  if (rc) return rc;
  k_advance_time<<<1, 1, 0, c->stream>>>(c->ds); MAC_COUNT(c);
  rc = check(cudaGetLastError());
  return rc ? rc : ode;
}

// ------------------------------------------------------- drop-in CSC solver
// A symmetric matrix's CSC arrays read as CSR rows: y_j = sum_k value[k] *
// x[indice[k]] over column j (the CG path; mac_csc_factorize checks symmetry).
__global__ void k_csc_spmv(int n, const int* __restrict__ off, const int* __restrict__ ind,
                           const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y,
                           double* partial_dot, const double* __restrict__ pdot) {
  double acc = 0;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    double s = 0;
    for (int k = off[j]; k < off[j + 1]; ++k) s += val[k] * x[ind[k]];
    s = -s;  // M = -A
    y[j] = s;
    acc += pdot[j] * s;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(partial_dot, acc);
}

__global__ void k_csc_diag(int n, const int* __restrict__ off, const int* __restrict__ ind,
                           const double* __restrict__ val, double* dinv) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    double d = 0;
    for (int k = off[j]; k < off[j + 1]; ++k)
      if (ind[k] == j) d = -val[k];
    dinv[j] = d != 0 ? 1.0 / d : 0.0;
  }
}

// mode 0: r = -b, x = 0, z = dinv r, p = z, scal[0] += r.z, scal[1] += b.b
// mode 1: x += a p, r -= a q, scal[2] += r.r
// mode 2: z = dinv r, scal[0] += r.z
// mode 3: p = z + beta p
__global__ void k_csc_vec(int n, int mode, const double* b, double* x, double* r, double* z, double* p,
                          const double* q, const double* dinv, double* scal, double a) {
  double s0 = 0, s1 = 0;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    if (mode == 0) {
      double rv = -b[j];
      r[j] = rv;
      x[j] = 0;
      double zv = dinv[j] * rv;
      z[j] = zv;
      p[j] = zv;
      s0 += rv * zv;
      s1 += b[j] * b[j];
    } else if (mode == 1) {
      x[j] += a * p[j];
      double rv = r[j] - a * q[j];
      r[j] = rv;
      s0 += rv * rv;
    } else if (mode == 2) {
      double zv = dinv[j] * r[j];
      z[j] = zv;
      s0 += r[j] * zv;
    } else {
      p[j] = z[j] + a * p[j];
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_down_sync(0xffffffffu, s0, o);
    s1 += __shfl_down_sync(0xffffffffu, s1, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (mode == 0) {
      atomicAdd(scal + 0, s0);
      atomicAdd(scal + 1, s1);
    } else if (mode == 1) {
      atomicAdd(scal + 2, s0);
    } else if (mode == 2) {
      atomicAdd(scal + 0, s0);
    }
  }
}

// CG breakdown: p.q of zero, or not finite, means the direction carries no
// information (a singular or indefinite system, or a zero row with b != 0).
static inline bool cg_breakdown(double pq) { return !(pq != 0.0 && std::isfinite(pq)); }

static int csc_solve_cg(Ctx* c, const double* hb, double* hx) {
  int n = c->csc_n;
  cudaStream_t st = c->stream;
  double* v = c->csc_vec;
  double *b = v, *x = v + n, *r = v + 2 * (size_t)n, *z = v + 3 * (size_t)n, *p = v + 4 * (size_t)n,
         *q = v + 5 * (size_t)n, *dinv = v + 6 * (size_t)n, *scal = v + 7 * (size_t)n;
  int g = grid_for(n, 256);
  if (g > 1184) g = 1184;
  int rc = check(cudaMemcpyAsync(b, hb, 8 * (size_t)n, cudaMemcpyHostToDevice, st));
  if (rc) return rc;
  k_csc_diag<<<g, 256, 0, st>>>(n, c->csc_off, c->csc_ind, c->csc_val, dinv); MAC_COUNT(c);
  cudaMemsetAsync(scal, 0, 8 * 8, st);
  k_csc_vec<<<g, 256, 0, st>>>(n, 0, b, x, r, z, p, q, dinv, scal, 0); MAC_COUNT(c);
  double hs[8];
  cudaMemcpyAsync(hs, scal, 64, cudaMemcpyDeviceToHost, st);
  if ((rc = check(cudaStreamSynchronize(st)))) return rc;
  double rz = hs[0], bb = hs[1];
  double rtol = c->prm.rtol;
  int it = 0;
  double rr = bb;
  while (bb > 0 && it < c->prm.max_iters) {
    cudaMemsetAsync(scal, 0, 64, st);
    k_csc_spmv<<<g, 256, 0, st>>>(n, c->csc_off, c->csc_ind, c->csc_val, p, q, scal + 3, p); MAC_COUNT(c);
    cudaMemcpyAsync(hs, scal, 64, cudaMemcpyDeviceToHost, st);
    if ((rc = check(cudaStreamSynchronize(st)))) return rc;
    if (cg_breakdown(hs[3])) break;  // x keeps the last finite iterate
    double alpha = rz / hs[3];
    k_csc_vec<<<g, 256, 0, st>>>(n, 1, b, x, r, z, p, q, dinv, scal, alpha); MAC_COUNT(c);
    k_csc_vec<<<g, 256, 0, st>>>(n, 2, b, x, r, z, p, q, dinv, scal, 0); MAC_COUNT(c);
    cudaMemcpyAsync(hs, scal, 64, cudaMemcpyDeviceToHost, st);
    if ((rc = check(cudaStreamSynchronize(st)))) return rc;
    ++it;
    rr = hs[2];
    if (rr <= rtol * rtol * bb) break;
    double beta = hs[0] / rz;
    rz = hs[0];
    k_csc_vec<<<g, 256, 0, st>>>(n, 3, b, x, r, z, p, q, dinv, scal, beta); MAC_COUNT(c);
  }
  if ((rc = check(cudaMemcpyAsync(hx, x, 8 * (size_t)n, cudaMemcpyDeviceToHost, st)))) return rc;
  if ((rc = check(cudaStreamSynchronize(st)))) return rc;
  c->stats.iterations = it;
  c->stats.total_iterations += it;
  c->stats.solves += 1;
  c->stats.relres = bb > 0 ? std::sqrt(rr / bb) : 0.0;
  c->stats.unknowns = n;
  return (bb > 0 && !(rr <= rtol * rtol * bb)) ? MAC_ERR_NOT_CONVERGED : MAC_OK;
}

// ---- general (non-symmetric) matrices: Jacobi-preconditioned BiCGStab on
// the row-major copy built at factorisation. A x is a row-wise product, so
// every y_i is summed in a fixed order.
// y = A x with scal[0] += w0.y and, with yy, scal[1] += y.y (formed from the
// value just computed: y is never read back).
__global__ void k_csr_spmv_dot(int n, const int* __restrict__ off, const int* __restrict__ ind,
                               const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y,
                               const double* __restrict__ w0, int yy, double* scal) {
  double a0 = 0, a1 = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0;
    for (int k = off[i]; k < off[i + 1]; ++k) s += val[k] * x[ind[k]];
    y[i] = s;
    a0 += w0[i] * s;
    if (yy) a1 += s * s;
  }
  for (int o = 16; o > 0; o >>= 1) {
    a0 += __shfl_down_sync(0xffffffffu, a0, o);
    a1 += __shfl_down_sync(0xffffffffu, a1, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(scal, a0);
    if (yy) atomicAdd(scal + 1, a1);
  }
}

// The diagonal's inverse from the row-major copy (1 where the diagonal is 0).
__global__ void k_csr_dinv(int n, const int* __restrict__ off, const int* __restrict__ ind,
                           const double* __restrict__ val, double* dinv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double d = 0;
    for (int k = off[i]; k < off[i + 1]; ++k)
      if (ind[k] == i) d += val[k];
    dinv[i] = d != 0 ? 1.0 / d : 1.0;
  }
}

// BiCGStab vector steps (van der Vorst 1992, right preconditioning K = diag):
// mode 0: r = rh = b, x = 0, p = v = 0; scal[2] += b.b
// mode 1: p = r + beta (p - omega v); y = K^-1 p
// mode 2: s = r - alpha v; z = K^-1 s; scal[2] += s.s
// mode 3: x += alpha y + omega z; r = s - omega t; scal[2] += r.r, scal[3] += rh.r
__global__ void k_bicg_vec(int n, int mode, const double* __restrict__ b, double* x, double* r,
                           double* rh, double* p, double* v, double* y, double* s,
                           double* z, const double* __restrict__ t, const double* __restrict__ dinv, double* scal,
                           double alpha, double beta, double omega) {
  double a0 = 0, a1 = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (mode == 0) {
      const double bv = b[i];
      r[i] = bv;
      rh[i] = bv;
      x[i] = 0.0;
      p[i] = 0.0;
      v[i] = 0.0;
      a0 += bv * bv;
    } else if (mode == 1) {
      const double pv = r[i] + beta * (p[i] - omega * v[i]);
      p[i] = pv;
      y[i] = dinv[i] * pv;
    } else if (mode == 2) {
      const double sv = r[i] - alpha * v[i];
      s[i] = sv;
      z[i] = dinv[i] * sv;
      a0 += sv * sv;
    } else {
      x[i] += alpha * y[i] + omega * z[i];
      const double rv = s[i] - omega * t[i];
      r[i] = rv;
      a0 += rv * rv;
      a1 += rh[i] * rv;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    a0 += __shfl_down_sync(0xffffffffu, a0, o);
    a1 += __shfl_down_sync(0xffffffffu, a1, o);
  }
  if ((threadIdx.x & 31) == 0 && mode != 1) {
    atomicAdd(scal + 2, a0);
    if (mode == 3) atomicAdd(scal + 3, a1);
  }
}

static int csc_solve_bicgstab(Ctx* c, const double* hb, double* hx) {
  const int n = c->csc_n;
  const size_t N = (size_t)n;
  cudaStream_t st = c->stream;
  double* w = c->csc_vec;
  double *b = w, *x = w + N, *r = w + 2 * N, *rh = w + 3 * N, *p = w + 4 * N, *v = w + 5 * N, *y = w + 6 * N,
         *s = w + 7 * N, *z = w + 8 * N, *t = w + 9 * N, *dinv = w + 10 * N, *scal = w + 11 * N;
  int g = grid_for(n, 256);
  if (g > 1184) g = 1184;
  double hs[8];
  auto read = [&]() {
    int e = check(cudaMemcpyAsync(hs, scal, 64, cudaMemcpyDeviceToHost, st));
    return e ? e : check(cudaStreamSynchronize(st));
  };
  int rc = check(cudaMemcpyAsync(b, hb, 8 * N, cudaMemcpyHostToDevice, st));
  if (rc) return rc;
  k_csr_dinv<<<g, 256, 0, st>>>(n, c->csr_off, c->csr_ind, c->csr_val, dinv); MAC_COUNT(c);
  cudaMemsetAsync(scal, 0, 64, st);
  k_bicg_vec<<<g, 256, 0, st>>>(n, 0, b, x, r, rh, p, v, y, s, z, t, dinv, scal, 0, 0, 0); MAC_COUNT(c);
  if ((rc = read())) return rc;
  const double bb = hs[2], rtol2 = c->prm.rtol * c->prm.rtol;
  double rr = bb, rho = bb, rho_prev = 1.0, alpha = 1.0, omega = 1.0;
  int it = 0;
  bool first = true;
  while (bb > 0 && it < c->prm.max_iters) {
    const double beta = first ? 0.0 : (rho / rho_prev) * (alpha / omega);
    first = false;
    k_bicg_vec<<<g, 256, 0, st>>>(n, 1, b, x, r, rh, p, v, y, s, z, t, dinv, scal, 0, beta, omega); MAC_COUNT(c);
    cudaMemsetAsync(scal, 0, 64, st);
    k_csr_spmv_dot<<<g, 256, 0, st>>>(n, c->csr_off, c->csr_ind, c->csr_val, y, v, rh, 0, scal); MAC_COUNT(c);
    if ((rc = read())) return rc;
    const double rhv = hs[0];
    if (cg_breakdown(rhv)) break;
    alpha = rho / rhv;
    cudaMemsetAsync(scal, 0, 64, st);
    k_bicg_vec<<<g, 256, 0, st>>>(n, 2, b, x, r, rh, p, v, y, s, z, t, dinv, scal, alpha, 0, 0); MAC_COUNT(c);
    k_csr_spmv_dot<<<g, 256, 0, st>>>(n, c->csr_off, c->csr_ind, c->csr_val, z, t, s, 1, scal); MAC_COUNT(c);
    if ((rc = read())) return rc;
    const double ts = hs[0], tt = hs[1], ss = hs[2];
    ++it;
    if (ss <= rtol2 * bb || cg_breakdown(tt)) {
      // converged on the half step (or t = 0): x += alpha y, r = s
      k_bicg_vec<<<g, 256, 0, st>>>(n, 3, b, x, r, rh, p, v, y, s, z, t, dinv, scal, alpha, 0, 0); MAC_COUNT(c);
      rr = ss;
      break;
    }
    omega = ts / tt;
    cudaMemsetAsync(scal, 0, 64, st);
    k_bicg_vec<<<g, 256, 0, st>>>(n, 3, b, x, r, rh, p, v, y, s, z, t, dinv, scal, alpha, 0, omega); MAC_COUNT(c);
    if ((rc = read())) return rc;
    rr = hs[2];
    if (rr <= rtol2 * bb) break;
    rho_prev = rho;
    rho = hs[3];
    if (cg_breakdown(rho) || omega == 0.0) break;
  }
  if ((rc = check(cudaMemcpyAsync(hx, x, 8 * N, cudaMemcpyDeviceToHost, st)))) return rc;
  if ((rc = check(cudaStreamSynchronize(st)))) return rc;
  c->stats.iterations = it;
  c->stats.total_iterations += it;
  c->stats.solves += 1;
  c->stats.relres = bb > 0 ? std::sqrt(rr / bb) : 0.0;
  c->stats.unknowns = n;
  return (bb > 0 && !(rr <= rtol2 * bb)) ? MAC_ERR_NOT_CONVERGED : MAC_OK;
}

static int csc_solve(Ctx* c, const double* hb, double* hx) {
  if (c->csc_n <= 0) return MAC_OK;
  return c->csc_general ? csc_solve_bicgstab(c, hb, hx) : csc_solve_cg(c, hb, hx);
}

// Host-side checks of a CSC matrix at factorisation. csc_valid: offsets start
// at 0 and never decrease, row indices lie in [0, n). csc_symmetric_negdiag:
// the matrix equals its transpose entry by entry and every diagonal entry is
// negative, the form Algorithms_Solve_Pressure::Init_Iteration assembles
// (src/Algorithms_Solve_Pressure.h:103-136), whose negation CG can solve.
static bool csc_valid(int n, const int* off, const int* ind) {
  if (off[0] != 0) return false;
  for (int j = 0; j < n; ++j)
    if (off[j + 1] < off[j]) return false;
  for (int k = 0; k < off[n]; ++k)
    if (ind[k] < 0 || ind[k] >= n) return false;
  return true;
}

struct Entry {
  int i, j;
  double v;
  bool operator<(const Entry& o) const { return i != o.i ? i < o.i : (j != o.j ? j < o.j : v < o.v); }
  bool operator==(const Entry& o) const { return i == o.i && j == o.j && v == o.v; }
};

static bool csc_symmetric_negdiag(int n, const int* off, const int* ind, const double* val) {
  const int nnz = off[n];
  std::vector<Entry> a(nnz), at(nnz);
  std::vector<int> diag(n, 0);
  for (int j = 0; j < n; ++j)
    for (int k = off[j]; k < off[j + 1]; ++k) {
      a[k] = {ind[k], j, val[k]};
      at[k] = {j, ind[k], val[k]};
      if (ind[k] == j) {
        if (!(val[k] < 0)) return false;
        diag[j] += 1;
      }
    }
  for (int j = 0; j < n; ++j)
    if (diag[j] != 1) return false;
  std::sort(a.begin(), a.end());
  std::sort(at.begin(), at.end());
  return a == at;
}

// Row-major copy (CSR) of a CSC matrix, rows in column order.
static void csc_to_csr(int n, const int* off, const int* ind, const double* val, std::vector<int>& roff,
                       std::vector<int>& rind, std::vector<double>& rval) {
  const int nnz = off[n];
  roff.assign(n + 1, 0);
  for (int k = 0; k < nnz; ++k) roff[ind[k] + 1] += 1;
  for (int i = 0; i < n; ++i) roff[i + 1] += roff[i];
  rind.resize(nnz);
  rval.resize(nnz);
  std::vector<int> cur(roff.begin(), roff.end() - 1);
  for (int j = 0; j < n; ++j)
    for (int k = off[j]; k < off[j + 1]; ++k) {
      const int q = cur[ind[k]]++;
      rind[q] = j;
      rval[q] = val[k];
    }
}

}  // namespace mac

using mac::Ctx;

#define CTX_OR_FAIL()                        \
  Ctx* c = (Ctx*)ctx;                        \
  if (!c) return MAC_ERR_INVALID;            \
  cudaSetDevice(c->prm.device)

extern "C" {

int mac_initialize_maccell(void* ctx) {
  CTX_OR_FAIL();
  return mac::topo_initialize(c);
}
int mac_layer_initial_with_particle(void* ctx) {
  CTX_OR_FAIL();
  int rc = mac::topo_layer_initial(c);
  return rc ? rc : mac::read_scalars(c);
}
int mac_create_fluid_particle(void* ctx) {
  CTX_OR_FAIL();
  int rc = mac::topo_create_fluid(c);
  return rc ? rc : mac::read_scalars(c);
}
int mac_update_celltype_layer(void* ctx) {
  CTX_OR_FAIL();
  int rc = mac::topo_update_layer(c);
  return rc ? rc : mac::read_scalars(c);
}
int mac_delete_maccell(void* ctx) {
  CTX_OR_FAIL();
  int rc = mac::topo_delete(c);
  return rc ? rc : mac::read_scalars(c);
}
int mac_calculate_time_step(void* ctx, double* dt) {
  CTX_OR_FAIL();
  int rc = mac::topo_dt(c);
  if (rc) return rc;
  rc = mac::topo_finish(c);
  if (dt) *dt = c->hs->dt;
  return rc;
}
int mac_topology_rebuild(void* ctx) {
  CTX_OR_FAIL();
  return mac::topology_rebuild(c, false);
}
int mac_forces(void* ctx, int ispeed) {
  CTX_OR_FAIL();
  if (ispeed < 0 || ispeed > 1) return MAC_ERR_INVALID;
  return mac::forces(c, ispeed);
}
int mac_pressure_project(void* ctx, int ispeed) {
  CTX_OR_FAIL();
  if (ispeed < 0 || ispeed > 1) return MAC_ERR_INVALID;
  int rc = mac::setup_system(c);
  return rc ? rc : mac::project(c, ispeed);
}
int mac_pressure_init(void* ctx) {
  CTX_OR_FAIL();
  return mac::setup_system(c);
}
int mac_pressure_divergence_projection(void* ctx, int ispeed, int accel) {
  CTX_OR_FAIL();
  if (ispeed < 0 || ispeed > 1 || (accel != 0 && accel != 1)) return MAC_ERR_INVALID;
  if (!c->system_ready) return MAC_ERR_INVALID;  // mac_pressure_init first
  const size_t cap = (size_t)c->cap_bricks * mac::kCells;
  double* S[3];
  double* A[3];
  for (int i = 0; i < 3; ++i) {
    S[i] = c->f64 + (size_t)(mac::U0X + 3 * ispeed + i) * cap;
    A[i] = c->f64 + (size_t)(mac::AX + i) * cap;
  }
  return accel ? mac::project_field(c, A, S) : mac::project_field(c, S, S);
}
int mac_pressure_end(void* ctx) {
  CTX_OR_FAIL();
  c->system_ready = false;
  return MAC_OK;
}
int mac_rk2tvd(void* ctx) {
  CTX_OR_FAIL();
  return mac::rk2tvd(c);
}
int mac_rungekutta_all(void* ctx) {
  CTX_OR_FAIL();
  return mac::rk_all(c);
}
int mac_extrapolate(void* ctx) {
  CTX_OR_FAIL();
  return mac::extrapolate(c);
}
int mac_move_particles(void* ctx) {
  CTX_OR_FAIL();
  return mac::move_particles(c);
}
int mac_step(void* ctx) {
  CTX_OR_FAIL();
  return mac::step(c);
}

int mac_set_preconditioner_net(void* ctx, void* net) {
  CTX_OR_FAIL();
  c->unet = net;
  return MAC_OK;
}

int mac_set_learned_smoothing(void* ctx, double omega) {
  CTX_OR_FAIL();
  if (!(omega >= 0.0 && omega < 2.0)) return MAC_ERR_INVALID;
  c->learned_omega = omega;
  return MAC_OK;
}

int mac_set_multigrid(void* ctx, int sweeps0, int prefetch) {
  CTX_OR_FAIL();
  if ((sweeps0 != 1 && sweeps0 != 2) || (prefetch != 0 && prefetch != 1)) return MAC_ERR_INVALID;
  c->mg_sweeps0 = sweeps0;
  c->mg_bulk = prefetch;
  return MAC_OK;
}

int mac_set_coarse_block(void* ctx, int max_cells) {
  CTX_OR_FAIL();
  if (max_cells < 64) return MAC_ERR_INVALID;
  c->blk_max_cells = max_cells;
  c->system_ready = false;  // the level split is made with the system
  return MAC_OK;
}

int mac_set_concurrent_binning(void* ctx, int on) {
  CTX_OR_FAIL();
  if (on != 0 && on != 1) return MAC_ERR_INVALID;
  c->bin_side = on;
  return MAC_OK;
}

int mac_set_dependent_launch(void* ctx, int on) {
  CTX_OR_FAIL();
  if (on != 0 && on != 1) return MAC_ERR_INVALID;
  c->pdl = on;
  return MAC_OK;
}

int mac_set_smoother(void* ctx, double w1, double w2, double w_single, double coarse_scale) {
  CTX_OR_FAIL();
  if (!(w1 > 0 && w1 < 4 && w2 > 0 && w2 < 4 && w_single > 0 && w_single < 1 && coarse_scale > 0 &&
        coarse_scale <= 1))
    return MAC_ERR_INVALID;
  // two sweeps damp lambda in (0, 2] by (1 - w1 lambda)(1 - w2 lambda): keep it inside (-1, 1)
  for (int k = 1; k <= 200; ++k) {
    const double l = 0.01 * k, f = (1 - w1 * l) * (1 - w2 * l);
    if (!(f > -1 && f < 1)) return MAC_ERR_INVALID;
  }
  c->dp.mgw1 = w1;
  c->dp.mgw2 = w2;
  c->dp.mgws = w_single;
  if (coarse_scale != c->mg_scale) {
    c->mg_scale = coarse_scale;
    c->system_ready = false;
  }
  return MAC_OK;
}

int mac_csc_factorize(void* ctx, int n, const int* offset, const int* indice, const double* value) {
  CTX_OR_FAIL();
  if (n < 0 || (n > 0 && (!offset || !indice || !value))) return MAC_ERR_INVALID;
  mac_csc_clean(ctx);
  if (n == 0) return MAC_OK;
  if (!mac::csc_valid(n, offset, indice)) return MAC_ERR_INVALID;
  int nnz = offset[n];
  // The reference's pressure matrix (symmetric, negative diagonal) goes to
  // Jacobi-CG; any other matrix Policy_Solve_Linear_Umfpack would factorise
  // goes to Jacobi-BiCGStab on a row-major copy.
  const bool general = !mac::csc_symmetric_negdiag(n, offset, indice, value);
  const size_t nvec = general ? 11 : 7;
  int rc = mac::check(cudaMalloc((void**)&c->csc_off, 4 * (size_t)(n + 1)));
  if (!rc) rc = mac::check(cudaMalloc((void**)&c->csc_ind, 4 * (size_t)(nnz ? nnz : 1)));
  if (!rc) rc = mac::check(cudaMalloc((void**)&c->csc_val, 8 * (size_t)(nnz ? nnz : 1)));
  if (!rc) rc = mac::check(cudaMalloc((void**)&c->csc_vec, 8 * (size_t)(nvec * (size_t)n + 8)));
  if (!rc) rc = mac::check(cudaMemcpyAsync(c->csc_off, offset, 4 * (size_t)(n + 1), cudaMemcpyHostToDevice, c->stream));
  if (!rc) rc = mac::check(cudaMemcpyAsync(c->csc_ind, indice, 4 * (size_t)nnz, cudaMemcpyHostToDevice, c->stream));
  if (!rc) rc = mac::check(cudaMemcpyAsync(c->csc_val, value, 8 * (size_t)nnz, cudaMemcpyHostToDevice, c->stream));
  std::vector<int> roff, rind;
  std::vector<double> rval;
  if (general && !rc) {
    mac::csc_to_csr(n, offset, indice, value, roff, rind, rval);
    rc = mac::check(cudaMalloc((void**)&c->csr_off, 4 * (size_t)(n + 1)));
    if (!rc) rc = mac::check(cudaMalloc((void**)&c->csr_ind, 4 * (size_t)(nnz ? nnz : 1)));
    if (!rc) rc = mac::check(cudaMalloc((void**)&c->csr_val, 8 * (size_t)(nnz ? nnz : 1)));
    if (!rc) rc = mac::check(cudaMemcpyAsync(c->csr_off, roff.data(), 4 * (size_t)(n + 1), cudaMemcpyHostToDevice, c->stream));
    if (!rc) rc = mac::check(cudaMemcpyAsync(c->csr_ind, rind.data(), 4 * (size_t)nnz, cudaMemcpyHostToDevice, c->stream));
    if (!rc) rc = mac::check(cudaMemcpyAsync(c->csr_val, rval.data(), 8 * (size_t)nnz, cudaMemcpyHostToDevice, c->stream));
  }
  if (!rc) rc = mac::check(cudaStreamSynchronize(c->stream));
  if (rc) {
    mac_csc_clean(ctx);
    return rc;
  }
  c->csc_n = n;
  c->csc_general = general ? 1 : 0;
  return MAC_OK;
}

int mac_csc_solve(void* ctx, int n, const double* b, double* x) {
  CTX_OR_FAIL();
  if (n != c->csc_n || (n > 0 && (!b || !x))) return MAC_ERR_INVALID;
  return mac::csc_solve(c, b, x);
}

int mac_csc_clean(void* ctx) {
  CTX_OR_FAIL();
  cudaFree(c->csc_off);
  cudaFree(c->csc_ind);
  cudaFree(c->csc_val);
  cudaFree(c->csc_vec);
  cudaFree(c->csr_off);
  cudaFree(c->csr_ind);
  cudaFree(c->csr_val);
  c->csr_off = nullptr;
  c->csr_ind = nullptr;
  c->csr_val = nullptr;
  c->csc_general = 0;
  c->csc_off = nullptr;
  c->csc_ind = nullptr;
  c->csc_val = nullptr;
  c->csc_vec = nullptr;
  c->csc_n = 0;
  return MAC_OK;
}

}  // extern "C"
