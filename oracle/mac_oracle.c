/* CPU restatement of Mac's per-timestep hot path (test infrastructure only).
 *
 * This is the oracle the CUDA path is checked against. It restates, in plain
 * C, the algorithms the reference composes in test/TestJetDEau_Basic.cpp:433-446
 * (pipeline A): topology rebuild, CFL time step, gravity + first-order upwind
 * convection, SSP-RK2 with two pressure projections, air-layer velocity
 * extrapolation and RK4 particle moves through the staggered trilinear field.
 * Every function cites the reference lines it follows. Arithmetic is written
 * in the reference's operation order (contraction off) so that non-solver
 * results agree bit for bit with the reference compiled from its own headers
 * (oracle/_ref/mac_ref, built by oracle/Makefile); the linear solve is FP64
 * Jacobi-CG to a relative residual of 1e-14 (the reference's Umfpack LU,
 * src/Policy_Solve_Linear_Umfpack.h:23-70, is not installed here).
 *
 * Only the tests, the smoke check and bench.py's CPU-baseline leg may load this
 * library, and only as a checker or a reported baseline.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "solve3.h"
#include "state_format.h"

#define ACC 3 /* index of the acceleration among the brick's vector fields */

typedef struct {
  int32_t key[3];
  uint8_t exists[512];
  double u[4][3][512]; /* speed buffers 0..2 and, at index ACC, the acceleration */
  double p[512];
  uint8_t flags[512];
  uint8_t type[512];
  int32_t layer[512];
  int32_t id[512];
  int32_t depth[512]; /* Data_Grid_Depth_Empty: -1 = empty */
  int32_t mark[512]; /* scratch */
} brick_t;

typedef struct {
  mac_state_header hdr;
  double h[3], ih[3];
  brick_t** b;
  int64_t nb, capb;
  int64_t* hkeys; /* open addressing table: packed key, -1 empty */
  int32_t* hval;
  int64_t hcap;
  double* pos;
  int64_t np, capp;
  uint64_t seed;
  int viscous; /* 1: Algorithms_Viscosity and the Dirichlet pressure are composed */
  /* Data_Chunk_Speed::ispeed (the speed buffer the stencils read) and
   * Data_Particle::imove_particle (the particle position the topology and the
   * interpolation use), src/Data_Chunk_Speed.h:17-19, src/Data_Particle.h:11-60;
   * pos1 / pos2 are the extra particle positions of pipeline B */
  int ispeed, imove;
  double *pos1, *pos2;
  /* statistics */
  int64_t invalid_reads, created_cells, cg_iters;
  double max_div, last_relres;
} world_t;

/* ------------------------------------------------------------------ grid */
static int64_t pack_key(int x, int y, int z) {
  return ((int64_t)(uint32_t)(x + (1 << 20)) & 0x1FFFFF) |
         (((int64_t)(uint32_t)(y + (1 << 20)) & 0x1FFFFF) << 21) |
         (((int64_t)(uint32_t)(z + (1 << 20)) & 0x1FFFFF) << 42);
}

static uint64_t hmix(uint64_t k) {
  k ^= k >> 33; k *= 0xff51afd7ed558ccdull; k ^= k >> 33; k *= 0xc4ceb9fe1a85ec53ull; k ^= k >> 33;
  return k;
}

static void hash_rebuild(world_t* w) {
  int64_t need = 64;
  while (need < 4 * (w->nb + 1)) need <<= 1;
  if (need != w->hcap) {
    free(w->hkeys); free(w->hval);
    w->hcap = need;
    w->hkeys = (int64_t*)malloc(sizeof(int64_t) * need);
    w->hval = (int32_t*)malloc(sizeof(int32_t) * need);
  }
  for (int64_t i = 0; i < w->hcap; ++i) w->hkeys[i] = -1;
  for (int64_t i = 0; i < w->nb; ++i) {
    int64_t k = pack_key(w->b[i]->key[0], w->b[i]->key[1], w->b[i]->key[2]);
    uint64_t s = hmix((uint64_t)k) & (uint64_t)(w->hcap - 1);
    while (w->hkeys[s] != -1) s = (s + 1) & (uint64_t)(w->hcap - 1);
    w->hkeys[s] = k;
    w->hval[s] = (int32_t)i;
  }
}

static int64_t brick_find(const world_t* w, int bx, int by, int bz) {
  int64_t k = pack_key(bx, by, bz);
  uint64_t s = hmix((uint64_t)k) & (uint64_t)(w->hcap - 1);
  while (w->hkeys[s] != -1) {
    if (w->hkeys[s] == k) return w->hval[s];
    s = (s + 1) & (uint64_t)(w->hcap - 1);
  }
  return -1;
}

/* Floor division of a cell key by the chunk edge (src/ChunkHashTable.tpp:180-196). */
static int fdiv8(int v) { return v >= 0 ? v / 8 : (v + 1) / 8 - 1; }
/* Offset x + 8y + 64z inside the chunk (src/Offset.h:14-24). */
static int offs(int x, int y, int z) { return (x & 7) + 8 * (y & 7) + 64 * (z & 7); }

static void brick_prototype(brick_t* b, int bx, int by, int bz) {
  memset(b, 0, sizeof(*b));
  b->key[0] = bx; b->key[1] = by; b->key[2] = bz;
  for (int o = 0; o < 512; ++o) { b->layer[o] = -1; b->id[o] = -1; b->depth[o] = -1; }
}

static int64_t brick_create(world_t* w, int bx, int by, int bz) {
  if (w->nb == w->capb) {
    w->capb = w->capb ? 2 * w->capb : 64;
    w->b = (brick_t**)realloc(w->b, sizeof(brick_t*) * w->capb);
  }
  brick_t* b = (brick_t*)malloc(sizeof(brick_t));
  brick_prototype(b, bx, by, bz);
  w->b[w->nb] = b;
  ++w->nb;
  if (4 * (w->nb + 1) > w->hcap) hash_rebuild(w);
  else {
    int64_t k = pack_key(bx, by, bz);
    uint64_t s = hmix((uint64_t)k) & (uint64_t)(w->hcap - 1);
    while (w->hkeys[s] != -1) s = (s + 1) & (uint64_t)(w->hcap - 1);
    w->hkeys[s] = k;
    w->hval[s] = (int32_t)(w->nb - 1);
  }
  return w->nb - 1;
}

typedef struct { int64_t b; int o; } cell_t;

/* Lookup without creation; b = -1 when the chunk does not exist. */
static cell_t cell_at(const world_t* w, int x, int y, int z) {
  cell_t c;
  c.b = brick_find(w, fdiv8(x), fdiv8(y), fdiv8(z));
  c.o = offs(x, y, z);
  return c;
}

static int cell_valid(const world_t* w, cell_t c) { return c.b >= 0 && w->b[c.b]->exists[c.o]; }

/* grid[key]: creates the chunk (from the prototype) and sets the existence bit
 * (src/ChunkHashTable.tpp:62-87). Data of a re-created cell is whatever the
 * chunk held. */
static cell_t cell_get(world_t* w, int x, int y, int z) {
  cell_t c = cell_at(w, x, y, z);
  if (c.b < 0) c.b = brick_create(w, fdiv8(x), fdiv8(y), fdiv8(z));
  if (!w->b[c.b]->exists[c.o]) ++w->created_cells;
  w->b[c.b]->exists[c.o] = 1;
  return c;
}

#define B(c) (w->b[(c).b])
static void key_of(const world_t* w, int64_t bi, int o, int k[3]) {
  k[0] = w->b[bi]->key[0] * 8 + (o & 7);
  k[1] = w->b[bi]->key[1] * 8 + ((o >> 3) & 7);
  k[2] = w->b[bi]->key[2] * 8 + (o >> 6);
}

/* Neighbour read helpers: a read of a cell that does not exist would
 * dereference a null chunk in the reference (src/Offset_Base_Neighbour.h:14-33);
 * here it returns the stored value (0 for a missing chunk) and is counted. */
static double rd_u(world_t* w, int ib, int i, const int k[3], int dx, int dy, int dz) {
  cell_t c = cell_at(w, k[0] + dx, k[1] + dy, k[2] + dz);
  if (!cell_valid(w, c)) ++w->invalid_reads;
  return c.b >= 0 ? B(c)->u[ib][i][c.o] : 0.0;
}
static double rd_p(world_t* w, const int k[3], int dx, int dy, int dz) {
  cell_t c = cell_at(w, k[0] + dx, k[1] + dy, k[2] + dz);
  if (!cell_valid(w, c)) ++w->invalid_reads;
  return c.b >= 0 ? B(c)->p[c.o] : 0.0;
}

/* GetIsFluid: Material_To_Type_Fluid(m) == Fluid, true for fluid, inflow and, in
 * the depth composition's cell type, interior
 * (src/Data_CellType_Fluid_Air_Solid_Inflow_Interior_0_Pres.tpp:24-44; the
 * 0-pressure material is never set by any algorithm). */
static int is_fluid(uint8_t t) { return t == MAC_FLUID || t == MAC_INFLOW || t == MAC_INTERIOR; }
/* Data_CellType_Domain_Fluid: in domain <=> GetIsFluid (src/Data_CellType_Domain_Fluid.h:59-62);
 * Data_CellType_Domain_Fluid_Without_0_Pres adds "and not 0-pressure"
 * (src/Data_CellType_Domain_Fluid_Without_0_Pres.h:59-62), the same here. */
static int in_domain(uint8_t t) { return is_fluid(t); }
/* Sticky setters (src/Data_CellType_Fluid_Air_Solid_Inflow.tpp:141-157; with the
 * interior material, src/Data_CellType_Fluid_Air_Solid_Inflow_Interior_0_Pres.tpp:217-249:
 * SetAir from fluid or interior, SetFluid from air or interior, SetInterior always). */
static uint8_t set_air(uint8_t t) { return (t == MAC_FLUID || t == MAC_INTERIOR) ? MAC_AIR : t; }
static uint8_t set_fluid(uint8_t t) { return (t == MAC_AIR || t == MAC_INTERIOR) ? MAC_FLUID : t; }

/* Data_Grid_Speed::Set(i, v, force) (src/Data_Grid_Speed.tpp:19-26): the three
 * buffers of a cell share its const bits (src/Data_Chunk_Speed.h:99-123). */
static void set_u(brick_t* b, double* arr, int o, int i, double v, int force) {
  if (force || !(b->flags[o] & (1u << i))) arr[o] = v;
}

/* ------------------------------------------------------------- topology */
/* src/Algorithms_Initialize_MacCell.h:15-21 */
static void alg_initialize(world_t* w) {
  for (int64_t bi = 0; bi < w->nb; ++bi)
    for (int o = 0; o < 512; ++o)
      if (w->b[bi]->exists[o]) w->b[bi]->layer[o] = -1;
}

/* Position buffer b of particle q. */
static double* pbuf(world_t* w, int b, int64_t q) { return (b == 0 ? w->pos : (b == 1 ? w->pos1 : w->pos2)) + 3 * q; }
/* The current position (Data_Particle::GetParticlePos with imove_particle). */
static double* ppos(world_t* w, int64_t q) { return pbuf(w, w->imove, q); }

/* Policy_Particle_To_Key::GetKeyFromParticle (src/Policy_Particle_To_Key.h:24-35). */
static void particle_key(const world_t* w, const double* pos, int k[3]) {
  for (int i = 0; i < 3; ++i) k[i] = (int)lround(pos[i] * w->ih[i]);
}

/* src/Algorithms_Layer_Initial_With_Particle.h:26-30 */
static void alg_layer_initial(world_t* w) {
  for (int64_t q = 0; q < w->np; ++q) {
    int k[3];
    particle_key(w, ppos(w, q), k);
    cell_t c = cell_get(w, k[0], k[1], k[2]);
    B(c)->layer[c.o] = 0;
    B(c)->type[c.o] = set_fluid(B(c)->type[c.o]);
  }
}

/* A new particle sets its current position only (src/Data_Particle.h:17-24);
 * the other buffers are written before they are read. */
static void add_particle(world_t* w, const double p[3]) {
  if (w->np == w->capp) {
    w->capp = w->capp ? 2 * w->capp : 1024;
    w->pos = (double*)realloc(w->pos, sizeof(double) * 3 * w->capp);
    w->pos1 = (double*)realloc(w->pos1, sizeof(double) * 3 * w->capp);
    w->pos2 = (double*)realloc(w->pos2, sizeof(double) * 3 * w->capp);
  }
  for (int b = 0; b < 3; ++b) memset(pbuf(w, b, w->np), 0, 24);
  memcpy(ppos(w, w->np), p, sizeof(double) * 3);
  ++w->np;
}

/* Erasing a particle keeps the order of the others in every buffer. */
static void particle_move(world_t* w, int64_t to, int64_t from) {
  if (to == from) return;
  for (int b = 0; b < 3; ++b) memmove(pbuf(w, b, to), pbuf(w, b, from), 24);
}

/* The refill policy's AddParticle(key): 8 jittered particles, or
 * Policy_Add_Particle_Cube(n) (src/Policy_Add_Particle_Cube.h:29-59): (2n+1)^3
 * particles at (k_i + t_i/(2n+1)) h_i, t_i = -n..n, x fastest. */
static void add_refill(world_t* w, const int k[3]) {
  const int n = w->hdr.refill_cube;
  if (n <= 0) {
    for (int s = 0; s < 8; ++s) {
      double p[3];
      mac_jitter8_position(w->seed, k[0], k[1], k[2], s, w->h[0], w->h[1], w->h[2], p);
      add_particle(w, p);
    }
    return;
  }
  const double dh = 1. / (2 * n + 1);
  int t[3] = {-n, -n, -n};
  while (1) {
    double p[3];
    for (int i = 0; i < 3; ++i) p[i] = (k[i] + t[i] * dh) * w->h[i];
    add_particle(w, p);
    int j = 0;
    while (j < 3 && t[j] >= n) { t[j] = -n; ++j; }
    if (j < 3) ++t[j];
    else break;
  }
}

/* src/Algorithms_Create_Fluid_Particle.h:25-33 with
 * Policy_Is_Inbound_Filling_Layer_CellType (src/Policy_Is_Inbound_Filling_Layer_CellType.h:16-19)
 * and the 8-jittered-particles refill. */
static void alg_create_fluid(world_t* w) {
  for (int64_t bi = 0; bi < w->nb; ++bi) {
    brick_t* b = w->b[bi];
    for (int o = 0; o < 512; ++o) {
      if (!b->exists[o] || b->type[o] != MAC_INFLOW || b->layer[o] != -1) continue;
      int k[3];
      key_of(w, bi, o, k);
      add_refill(w, k);
      b->layer[o] = 0;
      b->type[o] = set_fluid(b->type[o]);
    }
  }
}

/* ------------------------------------------------ depth composition
 * The topology passes of test/Jet3.cpp:519-549 (Policy_Depth(max, interior,
 * remove), src/Policy_Depth.h:12-26). */

/* src/Algorithms_Initialize_Layer_And_Depth.h:16-33: every cell's layer empty;
 * fluid cells that are not interior lose their depth. */
static void alg_initialize_depth(world_t* w) {
  for (int64_t bi = 0; bi < w->nb; ++bi) {
    brick_t* b = w->b[bi];
    for (int o = 0; o < 512; ++o) {
      if (!b->exists[o]) continue;
      b->layer[o] = -1;
      if (is_fluid(b->type[o]) && b->type[o] != MAC_INTERIOR) b->depth[o] = -1;
    }
  }
}

/* src/Algorithms_Layer_Initial_With_Particle_Depth.h:26-47: a particle in an
 * interior cell gives it layer 0 and is erased when the cell is deeper than the
 * removal depth; elsewhere layer 0 and SetFluid. The list keeps its order. */
static void alg_layer_initial_depth(world_t* w) {
  int64_t keep = 0;
  for (int64_t q = 0; q < w->np; ++q) {
    int k[3];
    particle_key(w, ppos(w, q), k);
    cell_t c = cell_get(w, k[0], k[1], k[2]);
    brick_t* b = B(c);
    int erase = 0;
    if (b->type[c.o] == MAC_INTERIOR) {
      b->layer[c.o] = 0;
      erase = b->depth[c.o] > w->hdr.depth_remove;
    } else {
      b->layer[c.o] = 0;
      b->type[c.o] = set_fluid(b->type[c.o]);
    }
    if (!erase) {
      particle_move(w, keep, q);
      ++keep;
    }
  }
  w->np = keep;
}

/* src/Algorithms_Create_Fluid_Particle_Depth.h:21-43: inflow cells still empty
 * are refilled (layer 0, SetFluid); empty interior cells no deeper than the
 * removal depth are refilled (layer 0); every other interior cell gets layer 0. */
static void alg_create_fluid_depth(world_t* w) {
  for (int64_t bi = 0; bi < w->nb; ++bi) {
    brick_t* b = w->b[bi];
    for (int o = 0; o < 512; ++o) {
      if (!b->exists[o]) continue;
      int k[3];
      key_of(w, bi, o, k);
      if (b->type[o] == MAC_INFLOW && b->layer[o] == -1) {
        add_refill(w, k);
        b->layer[o] = 0;
        b->type[o] = set_fluid(b->type[o]);
      } else if (b->type[o] == MAC_INTERIOR && b->layer[o] == -1 && b->depth[o] <= w->hdr.depth_remove) {
        add_refill(w, k);
        b->layer[o] = 0;
      } else if (b->type[o] == MAC_INTERIOR) {
        b->layer[o] = 0;
      }
    }
  }
}

static const int DIRS[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};

typedef struct { int* k; int64_t n, cap; } keylist;
static void kl_push(keylist* l, const int k[3]) {
  if (l->n == l->cap) { l->cap = l->cap ? 2 * l->cap : 256; l->k = (int*)realloc(l->k, sizeof(int) * 3 * l->cap); }
  memcpy(l->k + 3 * l->n, k, sizeof(int) * 3);
  ++l->n;
}

static int empty_or_invalid(world_t* w, int x, int y, int z) {
  cell_t c = cell_at(w, x, y, z);
  return !cell_valid(w, c) || B(c)->layer[c.o] == -1;
}

/* src/Algorithms_Update_CellType_Layer.h:22-89; with_depth: the depth form
 * src/Algorithms_Update_CellType_Layer_Depth.h:24-138, which first empties
 * every cell's depth and gives the seeds depth 0, then after the air layers
 * runs a BFS inward over layer-0 cells: depth d < DepthInterior -> SetFluid,
 * else SetInterior (seeds keep their material). */
static void alg_update_layer_depth_bfs(world_t* w, keylist* sback);
static void alg_update_layer_impl(world_t* w, int with_depth) {
  keylist s = {0}, s2 = {0}, sback = {0};
  int lmax = w->hdr.layer_max;
  for (int64_t bi = 0; bi < w->nb; ++bi)
    for (int o = 0; o < 512; ++o) {
      if (!w->b[bi]->exists[o]) continue;
      if (with_depth) w->b[bi]->depth[o] = -1;
      if (w->b[bi]->layer[o] != 0) continue;
      int k[3];
      key_of(w, bi, o, k);
      for (int d = 0; d < 6; ++d)
        if (empty_or_invalid(w, k[0] + DIRS[d][0], k[1] + DIRS[d][1], k[2] + DIRS[d][2])) {
          kl_push(&s, k);
          if (with_depth) {
            w->b[bi]->depth[o] = 0;
            kl_push(&sback, k);
          }
          break;
        }
    }
  for (int lay = 1; lay <= lmax; ++lay) {
    for (int64_t q = 0; q < s.n; ++q) {
      int* k = s.k + 3 * q;
      for (int d = 0; d < 6; ++d) {
        int x = k[0] + DIRS[d][0], y = k[1] + DIRS[d][1], z = k[2] + DIRS[d][2];
        if (empty_or_invalid(w, x, y, z)) {
          cell_t c = cell_get(w, x, y, z);
          B(c)->layer[c.o] = lay;
          B(c)->type[c.o] = set_air(B(c)->type[c.o]);
          int kk[3] = {x, y, z};
          kl_push(&s2, kk);
        }
      }
    }
    keylist t = s; s = s2; s2 = t; s2.n = 0;
  }
  for (int64_t q = 0; q < s.n; ++q) {
    int* k = s.k + 3 * q;
    for (int i = 0; i < 3; ++i) {
      int x = k[0] + (i == 0), y = k[1] + (i == 1), z = k[2] + (i == 2);
      if (empty_or_invalid(w, x, y, z)) {
        cell_t c = cell_get(w, x, y, z);
        B(c)->layer[c.o] = lmax + 1;
        B(c)->type[c.o] = set_air(B(c)->type[c.o]);
      }
    }
  }
  if (with_depth) alg_update_layer_depth_bfs(w, &sback);
  free(s.k); free(s2.k); free(sback.k);
}

static void alg_update_layer_depth_bfs(world_t* w, keylist* sback) {
  keylist s2 = {0};
  for (int depth = 1;; ++depth) {
    for (int64_t q = 0; q < sback->n; ++q) {
      int* k = sback->k + 3 * q;
      for (int d = 0; d < 6; ++d) {
        int x = k[0] + DIRS[d][0], y = k[1] + DIRS[d][1], z = k[2] + DIRS[d][2];
        cell_t c = cell_at(w, x, y, z);
        if (c.b < 0) continue; /* every neighbour of a layer-0 cell exists by now */
        brick_t* b = B(c);
        if (b->layer[c.o] != 0 || b->depth[c.o] != -1) continue;
        b->depth[c.o] = depth;
        b->type[c.o] = depth < w->hdr.depth_interior ? set_fluid(b->type[c.o]) : MAC_INTERIOR;
        int kk[3] = {x, y, z};
        kl_push(&s2, kk);
      }
    }
    keylist t = *sback; *sback = s2; s2 = t; s2.n = 0;
    if (sback->n == 0) break;
  }
  free(s2.k);
}

static void alg_update_layer(world_t* w) { alg_update_layer_impl(w, 0); }
static void alg_update_layer_depth(world_t* w) { alg_update_layer_impl(w, 1); }

/* src/Algorithms_Delete_MacCell.h:22-44 and chunk freeing in erase
 * (src/ChunkHashTable.tpp:132-147). */
static void alg_delete(world_t* w) {
  int64_t keep = 0;
  for (int64_t bi = 0; bi < w->nb; ++bi) {
    brick_t* b = w->b[bi];
    int any = 0;
    for (int o = 0; o < 512; ++o) {
      if (b->exists[o] && b->layer[o] == -1 && !(b->flags[o] & MAC_FLAG_NODELETE)) b->exists[o] = 0;
      any |= b->exists[o];
    }
    if (any) w->b[keep++] = b;
    else free(b);
  }
  w->nb = keep;
  hash_rebuild(w);
}

/* src/Algorithms_Calculate_Time_Step.h:41-62 and src/Policy_CheckDT.h:16-29 */
static void alg_dt(world_t* w) {
  double mx = 0;
  for (int64_t bi = 0; bi < w->nb; ++bi)
    for (int o = 0; o < 512; ++o) {
      brick_t* b = w->b[bi];
      if (!b->exists[o] || !is_fluid(b->type[o])) continue;
      double t = 0;
      for (int i = 0; i < 3; ++i) {
        double v = b->u[0][i][o] * w->ih[i];
        t += v * v;
      }
      if (t > mx) mx = t;
    }
  double dt = 1 / sqrt(mx) * w->hdr.cfl_factor;
  if (dt < w->hdr.dt_min) dt = w->hdr.dt_min;
  else if (dt > w->hdr.dt_max) dt = w->hdr.dt_max;
  w->hdr.dt = dt;
}

/* ------------------------------------------------------------- advection */
/* Policy_Gravity::NeedToApply / ApplyGravity (src/Policy_Gravity.h:14-45). */
static void alg_gravity(world_t* w, int ib) {
  (void)ib;
  int ax = w->hdr.gravity_axis - 1;
  for (int64_t bi = 0; bi < w->nb; ++bi) {
    brick_t* b = w->b[bi];
    for (int o = 0; o < 512; ++o) {
      if (!b->exists[o]) continue;
      int apply = 0;
      if (is_fluid(b->type[o])) apply = 1;
      else if (b->layer[o] != -1) {
        int k[3];
        key_of(w, bi, o, k);
        k[ax] -= 1;
        cell_t n = cell_at(w, k[0], k[1], k[2]);
        apply = cell_valid(w, n) && is_fluid(B(n)->type[n.o]);
      }
      if (apply) set_u(b, b->u[ACC][ax], o, ax, b->u[ACC][ax][o] + w->hdr.gravity, 0);
    }
  }
}

/* Policy_Convection_Apply_If::Get_If_Apply_Convection(neigh, i)
 * (src/Policy_Convection_Apply_If.h:41-61). */
static int conv_apply(world_t* w, int64_t bi, int o, int i) {
  brick_t* b = w->b[bi];
  if (is_fluid(b->type[o])) return 1;
  if (b->layer[o] == -1) return 0;
  int k[3];
  key_of(w, bi, o, k);
  k[i] -= 1;
  cell_t n = cell_at(w, k[0], k[1], k[2]);
  if (!cell_valid(w, n)) return 0;
  return is_fluid(B(n)->type[n.o]);
}

/* Get_Speed_At_Bound (src/Policy_Speed_Interpolation_Linear_Symmetric.h:120-127). */
static double speed_at_bound(world_t* w, int ib, const int k[3], int i, int j) {
  if (i == j) return rd_u(w, ib, j, k, 0, 0, 0);
  int ej[3] = {0, 0, 0}, ei[3] = {0, 0, 0};
  ej[j] = 1; ei[i] = 1;
  double a = rd_u(w, ib, j, k, 0, 0, 0);
  double b = rd_u(w, ib, j, k, ej[0], ej[1], ej[2]);
  double c = rd_u(w, ib, j, k, -ei[0], -ei[1], -ei[2]);
  double d = rd_u(w, ib, j, k, ej[0] - ei[0], ej[1] - ei[1], ej[2] - ei[2]);
  return 0.25 * (((a + b) + c) + d);
}

/* Policy_Upwind_1_Order::Get_Convection_Element / Get_Convection_Speed
 * (src/Policy_Upwind_1_Order.h:18-38,58-66). */
static double convection_speed(world_t* w, int ib, const int k[3], int i) {
  double ret = 0;
  for (int j = 0; j < 3; ++j) {
    double U = speed_at_bound(w, ib, k, i, j);
    int e[3] = {0, 0, 0};
    e[j] = 1;
    double U1 = rd_u(w, ib, i, k, 0, 0, 0), U2;
    if (U > 0) {
      U2 = rd_u(w, ib, i, k, -e[0], -e[1], -e[2]);
      U *= (U1 - U2) * w->ih[j];
    } else {
      U2 = rd_u(w, ib, i, k, e[0], e[1], e[2]);
      U *= (U2 - U1) * w->ih[j];
    }
    ret -= U;
  }
  return ret;
}

/* src/Algorithms_Convection.h:24-33 */
static void alg_convection(world_t* w, int ib) {
  for (int64_t bi = 0; bi < w->nb; ++bi) {
    brick_t* b = w->b[bi];
    for (int o = 0; o < 512; ++o) {
      if (!b->exists[o]) continue;
      int k[3];
      key_of(w, bi, o, k);
      for (int i = 0; i < 3; ++i)
        if (conv_apply(w, bi, o, i)) set_u(b, b->u[ACC][i], o, i, b->u[ACC][i][o] + convection_speed(w, ib, k, i), 0);
    }
  }
}

/* Policy_Viscosity_Apply_If::Get_If_Apply_Viscosity (src/Policy_Viscosity_Apply_If.h:17-38). */
static int visc_apply(world_t* w, int64_t bi, int o) {
  brick_t* b = w->b[bi];
  if (is_fluid(b->type[o])) return 1;
  if (b->layer[o] == -1) return 0;
  int k[3];
  key_of(w, bi, o, k);
  for (int i = 0; i < 3; ++i) {
    int m[3] = {k[0], k[1], k[2]};
    m[i] -= 1;
    cell_t n = cell_at(w, m[0], m[1], m[2]);
    if (!cell_valid(w, n)) continue;
    if (is_fluid(B(n)->type[n.o])) return 1;
  }
  return 0;
}

/* Algorithms_Viscosity::Do (src/Algorithms_Viscosity.h:24-30) with
 * Policy_Laplacian_Speed::Get_Laplacian_Speed (src/Policy_Laplacian_Speed.h:22-36):
 * acc += viscosity * (sum_j u_i(c+e_j) + u_i(c-e_j) - 2 u_i(c)) / h_j^2, through
 * the non-forced Set, in the reference's summation order. */
static void alg_viscosity(world_t* w, int ib) {
  const double nu = w->hdr.viscosity;
  for (int64_t bi = 0; bi < w->nb; ++bi) {
    brick_t* b = w->b[bi];
    for (int o = 0; o < 512; ++o) {
      if (!b->exists[o] || !visc_apply(w, bi, o)) continue;
      int k[3];
      key_of(w, bi, o, k);
      double lap[3];
      for (int i = 0; i < 3; ++i) {
        double temp = 0;
        for (int j = 0; j < 3; ++j) {
          const double ih2 = pow(w->ih[j], 2);
          temp -= 2 * rd_u(w, ib, i, k, 0, 0, 0) * ih2;
          temp += rd_u(w, ib, i, k, j == 0, j == 1, j == 2) * ih2;
          temp += rd_u(w, ib, i, k, -(j == 0), -(j == 1), -(j == 2)) * ih2;
        }
        lap[i] = temp;
      }
      for (int i = 0; i < 3; ++i) set_u(b, b->u[ACC][i], o, i, b->u[ACC][i][o] + lap[i] * nu, 0);
    }
  }
}

/* Gravity, convection and, in the viscous composition, viscosity. */
static void grid_forces(world_t* w, int ib) {
  alg_gravity(w, ib);
  alg_convection(w, ib);
  if (w->viscous) alg_viscosity(w, ib);
}

static void acc_zero(world_t* w) {
  for (int64_t bi = 0; bi < w->nb; ++bi)
    for (int o = 0; o < 512; ++o)
      if (w->b[bi]->exists[o])
        for (int i = 0; i < 3; ++i) w->b[bi]->u[ACC][i][o] = 0.0;
}

/* ------------------------------------------------------------- pressure */
typedef struct {
  int64_t n;
  int64_t* rowptr;
  int64_t* col;
  double* val;
  double* diag;
  int64_t* bi; /* cell of each unknown */
  int* o;
} csr_t;

static void csr_free(csr_t* A) { free(A->rowptr); free(A->col); free(A->val); free(A->diag); free(A->bi); free(A->o); memset(A, 0, sizeof(*A)); }

/* Von Neumann face test: GetIsConstantInterface_Impl(neigh, dim, sign)
 * (src/Data_CellType_Interface_Constant.h:45-61). */
static int neumann(world_t* w, cell_t c, cell_t n, int i, int s) {
  if (!cell_valid(w, n)) return 0;
  return s > 0 ? (B(n)->flags[n.o] >> i) & 1 : (B(c)->flags[c.o] >> i) & 1;
}

/* Assembly of the ghost-fluid 7-point matrix (src/Algorithms_Solve_Pressure.h:44-157):
 * diag -= 1/h^2 per face, += 1/h^2 back on a valid Neumann face, off-diagonal
 * +1/h^2 to a valid in-domain neighbour; anything else is Dirichlet p = 0.
 * Unknowns are numbered in brick order rather than by the reference's BFS; the
 * solution of the system does not depend on the numbering. */
static void assemble(world_t* w, csr_t* A) {
  memset(A, 0, sizeof(*A));
  int64_t n = 0;
  for (int64_t bi = 0; bi < w->nb; ++bi)
    for (int o = 0; o < 512; ++o) {
      brick_t* b = w->b[bi];
      b->id[o] = -1;
      if (b->exists[o] && in_domain(b->type[o])) b->id[o] = (int32_t)n++;
    }
  A->n = n;
  A->rowptr = (int64_t*)calloc(n + 1, 8);
  A->col = (int64_t*)malloc(sizeof(int64_t) * (6 * n + 1));
  A->val = (double*)malloc(sizeof(double) * (6 * n + 1));
  A->diag = (double*)malloc(sizeof(double) * (n + 1));
  A->bi = (int64_t*)malloc(sizeof(int64_t) * (n + 1));
  A->o = (int*)malloc(sizeof(int) * (n + 1));
  int64_t nnz = 0;
  for (int64_t bi = 0; bi < w->nb; ++bi)
    for (int o = 0; o < 512; ++o) {
      brick_t* b = w->b[bi];
      if (b->id[o] < 0) continue;
      int64_t r = b->id[o];
      A->bi[r] = bi; A->o[r] = o;
      int k[3];
      key_of(w, bi, o, k);
      cell_t c = {bi, o};
      double diag = 0;
      for (int i = 0; i < 3; ++i)
        for (int s = -1; s <= 1; s += 2) {
          double h2 = w->ih[i] * w->ih[i];
          diag -= h2;
          cell_t nb = cell_at(w, k[0] + s * (i == 0), k[1] + s * (i == 1), k[2] + s * (i == 2));
          if (!cell_valid(w, nb)) continue;
          if (neumann(w, c, nb, i, s)) diag += h2;
          else if (in_domain(B(nb)->type[nb.o])) {
            A->col[nnz] = B(nb)->id[nb.o];
            A->val[nnz] = h2;
            ++nnz;
          }
        }
      A->diag[r] = diag;
      A->rowptr[r + 1] = nnz;
    }
}

/* y = A x */
static void spmv(const csr_t* A, const double* x, double* y) {
  for (int64_t r = 0; r < A->n; ++r) {
    double s = A->diag[r] * x[r];
    for (int64_t k = A->rowptr[r]; k < A->rowptr[r + 1]; ++k) s += A->val[k] * x[A->col[k]];
    y[r] = s;
  }
}

static double g_rtol = 1e-14;

/* FP64 Jacobi-preconditioned CG on -A (SPD), standing in for the LU solve. */
static void solve(world_t* w, const csr_t* A, const double* b, double* x) {
  int64_t n = A->n;
  double *r = (double*)malloc(8 * (n + 1)), *z = (double*)malloc(8 * (n + 1)),
         *p = (double*)malloc(8 * (n + 1)), *q = (double*)malloc(8 * (n + 1));
  double bn = 0;
  for (int64_t i = 0; i < n; ++i) { x[i] = 0; r[i] = -b[i]; bn += b[i] * b[i]; }
  bn = sqrt(bn);
  w->last_relres = 0;
  if (bn > 0) {
    double rz = 0;
    for (int64_t i = 0; i < n; ++i) { z[i] = r[i] / -A->diag[i]; p[i] = z[i]; rz += r[i] * z[i]; }
    for (int it = 0; it < 200000; ++it) {
      spmv(A, p, q);
      double pq = 0;
      for (int64_t i = 0; i < n; ++i) { q[i] = -q[i]; pq += p[i] * q[i]; }
      double a = rz / pq, rn = 0;
      for (int64_t i = 0; i < n; ++i) { x[i] += a * p[i]; r[i] -= a * q[i]; rn += r[i] * r[i]; }
      ++w->cg_iters;
      w->last_relres = sqrt(rn) / bn;
      if (sqrt(rn) <= g_rtol * bn) break;
      double rz2 = 0;
      for (int64_t i = 0; i < n; ++i) { z[i] = r[i] / -A->diag[i]; rz2 += r[i] * z[i]; }
      double be = rz2 / rz;
      rz = rz2;
      for (int64_t i = 0; i < n; ++i) p[i] = z[i] + be * p[i];
    }
  }
  free(r); free(z); free(p); free(q);
}

/* Policy_Divergence::Get_Divergence (src/Policy_Divergence.h:20-29). */
static double divergence(world_t* w, int ib, const int k[3]) {
  double ret = 0;
  for (int i = 0; i < 3; ++i) {
    ret -= rd_u(w, ib, i, k, 0, 0, 0) * w->ih[i];
    ret += rd_u(w, ib, i, k, i == 0, i == 1, i == 2) * w->ih[i];
  }
  return ret;
}

/* Policy_Pressure_If_Correction::Get_Pressure_If_Correction(neigh, i)
 * (src/Policy_Pressure_If_Correction.h:33-49). */
static int correction_applies(world_t* w, int64_t bi, int o, int i) {
  if (in_domain(w->b[bi]->type[o])) return 1;
  int k[3];
  key_of(w, bi, o, k);
  k[i] -= 1;
  cell_t n = cell_at(w, k[0], k[1], k[2]);
  if (!cell_valid(w, n)) return 0;
  return in_domain(B(n)->type[n.o]);
}

/* Policy_Dirichlet_Boundary (src/Policy_Dirichlet_Boundary.h:27-109).
 * GetIsAir compares Material_To_Type_Fluid with Air, and that map sends
 * Solid to Air as well (src/Data_CellType_Fluid_Air_Solid_Inflow.tpp:21-35):
 * "air" here means air or solid. */
static int is_air(uint8_t t) { return t == MAC_AIR || t == MAC_SOLID; }

/* GetIsDirichletBoundary: an air cell with a non-air face neighbour. */
static int dir_boundary(world_t* w, const int k[3]) {
  cell_t c = cell_at(w, k[0], k[1], k[2]);
  if (!cell_valid(w, c) || !is_air(B(c)->type[c.o])) return 0;
  for (int i = 0; i < 3; ++i)
    for (int s = -1; s <= 1; s += 2) {
      cell_t n = cell_at(w, k[0] + s * (i == 0), k[1] + s * (i == 1), k[2] + s * (i == 2));
      if (cell_valid(w, n) && !is_air(B(n)->type[n.o])) return 1;
    }
  return 0;
}

/* GetDirichletBoundaryPressure: -sum over non-air face neighbours (i, s) of
 * 2 viscosity (u_i(c+e_i) - u_i(c)) / h_i * s, in the reference's order. */
static double dir_pressure(world_t* w, int ib, const int k[3]) {
  cell_t c = cell_at(w, k[0], k[1], k[2]);
  if (!cell_valid(w, c) || !is_air(B(c)->type[c.o])) return 0;
  const double nu = w->hdr.viscosity;
  double ret = 0;
  for (int i = 0; i < 3; ++i)
    for (int s = -1; s <= 1; s += 2) {
      cell_t n = cell_at(w, k[0] + s * (i == 0), k[1] + s * (i == 1), k[2] + s * (i == 2));
      if (cell_valid(w, n) && !is_air(B(n)->type[n.o])) {
        const double v1 = rd_u(w, ib, i, k, 0, 0, 0);
        const double v2 = rd_u(w, ib, i, k, i == 0, i == 1, i == 2);
        ret -= 2 * nu * (v2 - v1) * w->ih[i] * s;
      }
    }
  return ret;
}

/* GetDirichletSumBoundaryPressure: sum over Dirichlet face neighbours of p_D / h_i^2. */
static double dir_sum(world_t* w, int ib, const int k[3]) {
  double ret = 0;
  for (int i = 0; i < 3; ++i)
    for (int s = -1; s <= 1; s += 2) {
      int m[3] = {k[0] + s * (i == 0), k[1] + s * (i == 1), k[2] + s * (i == 2)};
      if (dir_boundary(w, m)) ret += dir_pressure(w, ib, m) * w->ih[i] * w->ih[i];
    }
  return ret;
}

/* Algorithms_Solve_Pressure::Divergence_Projection (src/Algorithms_Solve_Pressure.h:168-222)
 * on speed buffer ib with an already assembled system; in the viscous
 * composition Algorithms_Solve_Pressure_Dirichlet::Divergence_Projection
 * (src/Algorithms_Solve_Pressure_Dirichlet.h:171-233): b -= the Dirichlet sum,
 * and Dirichlet air cells take their boundary pressure. */
/* The projection of vector field f (a speed buffer, or ACC for the force
 * projection of Algorithms_Solve_Pressure_Force, src/Algorithms_Solve_Pressure_Force.h:16-24,
 * where Speed_GetRef() returns the acceleration); the Dirichlet pressures read
 * speed buffer idir (Speed_GetRef(-1, false), src/Policy_Dirichlet_Boundary.h:100-102). */
static void project_field(world_t* w, const csr_t* A, int f, int idir);
static void project_with(world_t* w, const csr_t* A, int ib) { project_field(w, A, ib, ib); }
static void project_field(world_t* w, const csr_t* A, int f, int idir) {
  const int ib = f;
  int64_t n = A->n;
  double* b = (double*)malloc(8 * (n + 1));
  double* x = (double*)malloc(8 * (n + 1));
  for (int64_t r = 0; r < n; ++r) {
    int k[3];
    key_of(w, A->bi[r], A->o[r], k);
    b[r] = divergence(w, ib, k);
    if (w->viscous) b[r] -= dir_sum(w, idir, k);
  }
  solve(w, A, b, x);
  for (int64_t bi = 0; bi < w->nb; ++bi)
    for (int o = 0; o < 512; ++o) {
      brick_t* br = w->b[bi];
      if (!br->exists[o]) continue;
      if (in_domain(br->type[o])) {
        br->p[o] = x[br->id[o]];
      } else if (w->viscous) {
        int k[3];
        key_of(w, bi, o, k);
        br->p[o] = dir_boundary(w, k) ? dir_pressure(w, idir, k) : 0.0;
      } else {
        br->p[o] = 0.0;
      }
    }
  for (int64_t bi = 0; bi < w->nb; ++bi)
    for (int o = 0; o < 512; ++o) {
      brick_t* br = w->b[bi];
      if (!br->exists[o]) continue;
      int k[3];
      key_of(w, bi, o, k);
      for (int i = 0; i < 3; ++i)
        if (correction_applies(w, bi, o, i)) {
          /* Policy_Gradiant::Get_Gradiant(neigh, i) (src/Policy_Gradiant.h:32-37) */
          double g = br->p[o] * w->ih[i];
          g -= rd_p(w, k, -(i == 0), -(i == 1), -(i == 2)) * w->ih[i];
          set_u(br, br->u[ib][i], o, i, br->u[ib][i][o] - g, 0);
        }
    }
  w->max_div = 0;
  for (int64_t r = 0; r < n; ++r) {
    int k[3];
    key_of(w, A->bi[r], A->o[r], k);
    double d = fabs(divergence(w, ib, k));
    if (d > w->max_div) w->max_div = d;
  }
  free(b); free(x);
}

/* src/Algorithms_RungeKutta_RK2_TVD.h:20-66 with Policy = Algorithms<Gravity,
 * Convection> + Algorithms_Solve_Pressure. */
static void alg_rk2(world_t* w) {
  csr_t A;
  assemble(w, &A);
  double dt = w->hdr.dt;
  acc_zero(w);
  grid_forces(w, 0);
  for (int64_t bi = 0; bi < w->nb; ++bi)
    for (int o = 0; o < 512; ++o) {
      brick_t* b = w->b[bi];
      if (!b->exists[o]) continue;
      for (int i = 0; i < 3; ++i) b->u[1][i][o] = b->u[0][i][o] + b->u[ACC][i][o] * dt;
    }
  acc_zero(w);
  project_with(w, &A, 1);
  grid_forces(w, 1);
  for (int64_t bi = 0; bi < w->nb; ++bi)
    for (int o = 0; o < 512; ++o) {
      brick_t* b = w->b[bi];
      if (!b->exists[o]) continue;
      for (int i = 0; i < 3; ++i) {
        double v = 0.5 * b->u[0][i][o] + 0.5 * b->u[1][i][o] + 0.5 * b->u[ACC][i][o] * dt;
        set_u(b, b->u[0][i], o, i, v, 0);
      }
    }
  project_with(w, &A, 0);
  csr_free(&A);
}

/* Algorithms_Do_Pressure::Do (src/Algorithms_Do_Pressure.h:16-21) on speed 0. */
static void alg_project(world_t* w) {
  csr_t A;
  assemble(w, &A);
  project_with(w, &A, 0);
  csr_free(&A);
}

/* ---------------------------------------------------------- extrapolation */
static int lay_of(world_t* w, int x, int y, int z, int* valid) {
  cell_t c = cell_at(w, x, y, z);
  *valid = cell_valid(w, c) && B(c)->layer[c.o] != -1;
  return *valid ? B(c)->layer[c.o] : -1;
}

/* Algorithms_Extrapolate::Do (src/Algorithms_Extrapolate.h:25-233): level by
 * level, each face between a layer-lay cell and a cell of layer >= lay (or a
 * missing one on the minus side) gets the mean of the parallel or collinear
 * faces that touch a lower layer. n == 0 yields 0/0 as in the reference. */
static void alg_extrapolate_f(world_t* w, int fld) {
  keylist set = {0}, set2 = {0};
  for (int64_t bi = 0; bi < w->nb; ++bi)
    for (int o = 0; o < 512; ++o) {
      brick_t* b = w->b[bi];
      if (b->exists[o]) b->mark[o] = 0;
      if (b->exists[o] && b->layer[o] == 1) {
        int k[3];
        key_of(w, bi, o, k);
        kl_push(&set, k);
      }
    }
  int lay = 1;
  int gen = 1;
  while (1) {
    ++gen;
    for (int64_t q = 0; q < set.n; ++q) {
      int* K = set.k + 3 * q;
      for (int i = 0; i < 3; ++i) {
        int e[3] = {i == 0, i == 1, i == 2};
        int v2, v3, v4;
        /* +1 direction: face u_i(neigh2) with neigh2 = K + e_i */
        int l2 = lay_of(w, K[0] + e[0], K[1] + e[1], K[2] + e[2], &v2);
        if (v2 && l2 >= lay) {
          if (l2 > lay) {
            cell_t c2 = cell_at(w, K[0] + e[0], K[1] + e[1], K[2] + e[2]);
            if (B(c2)->mark[c2.o] != gen) {
              B(c2)->mark[c2.o] = gen;
              int kk[3] = {K[0] + e[0], K[1] + e[1], K[2] + e[2]};
              kl_push(&set2, kk);
            }
          }
          int n = 0;
          double val = 0;
          for (int j = 0; j < 3; ++j) {
            int f[3] = {j == 0, j == 1, j == 2};
            for (int s2 = -1; s2 <= 1; s2 += 2) {
              if (s2 == -1 && j == i) {
                int l3 = lay_of(w, K[0] - e[0], K[1] - e[1], K[2] - e[2], &v3);
                if (v3 && l3 < lay) { ++n; val += rd_u(w, fld, i, K, 0, 0, 0); }
              } else if (s2 == 1 && j == i) {
                int l3 = lay_of(w, K[0] + 2 * e[0], K[1] + 2 * e[1], K[2] + 2 * e[2], &v3);
                if (v3 && l3 < lay) { ++n; val += rd_u(w, fld, i, K, 2 * e[0], 2 * e[1], 2 * e[2]); }
              } else {
                int d3[3] = {e[0] + s2 * f[0], e[1] + s2 * f[1], e[2] + s2 * f[2]};
                int d4[3] = {s2 * f[0], s2 * f[1], s2 * f[2]};
                int l3 = lay_of(w, K[0] + d3[0], K[1] + d3[1], K[2] + d3[2], &v3);
                int l4 = lay_of(w, K[0] + d4[0], K[1] + d4[1], K[2] + d4[2], &v4);
                if (v3 && v4 && (l3 < lay || l4 < lay)) { ++n; val += rd_u(w, fld, i, K, d3[0], d3[1], d3[2]); }
              }
            }
          }
          cell_t c2 = cell_at(w, K[0] + e[0], K[1] + e[1], K[2] + e[2]);
          set_u(B(c2), B(c2)->u[fld][i], c2.o, i, val / n, 0);
        }
        /* -1 direction: face u_i(neigh) with neigh2 = K - e_i */
        l2 = lay_of(w, K[0] - e[0], K[1] - e[1], K[2] - e[2], &v2);
        cell_t c = cell_at(w, K[0], K[1], K[2]);
        if (v2) {
          if (l2 >= lay) {
            if (l2 > lay) {
              cell_t c2 = cell_at(w, K[0] - e[0], K[1] - e[1], K[2] - e[2]);
              if (B(c2)->mark[c2.o] != gen) {
                B(c2)->mark[c2.o] = gen;
                int kk[3] = {K[0] - e[0], K[1] - e[1], K[2] - e[2]};
                kl_push(&set2, kk);
              }
            }
            int n = 0;
            double val = 0;
            for (int j = 0; j < 3; ++j) {
              int f[3] = {j == 0, j == 1, j == 2};
              for (int s2 = -1; s2 <= 1; s2 += 2) {
                if (s2 == 1 && j == i) {
                  int l3 = lay_of(w, K[0] + f[0], K[1] + f[1], K[2] + f[2], &v3);
                  if (v3 && l3 < lay) { ++n; val += rd_u(w, fld, j, K, f[0], f[1], f[2]); }
                } else if (s2 == -1 && j == i) {
                  int l3 = lay_of(w, K[0] - 2 * f[0], K[1] - 2 * f[1], K[2] - 2 * f[2], &v3);
                  if (v3 && l3 < lay) { ++n; val += rd_u(w, fld, j, K, -f[0], -f[1], -f[2]); }
                } else {
                  int d3[3] = {-e[0] + s2 * f[0], -e[1] + s2 * f[1], -e[2] + s2 * f[2]};
                  int d4[3] = {s2 * f[0], s2 * f[1], s2 * f[2]};
                  int l3 = lay_of(w, K[0] + d3[0], K[1] + d3[1], K[2] + d3[2], &v3);
                  int l4 = lay_of(w, K[0] + d4[0], K[1] + d4[1], K[2] + d4[2], &v4);
                  if (v3 && v4 && (l3 < lay || l4 < lay)) { ++n; val += rd_u(w, fld, i, K, d4[0], d4[1], d4[2]); }
                }
              }
            }
            set_u(B(c), B(c)->u[fld][i], c.o, i, val / n, 0);
          }
        } else {
          int n = 0;
          double val = 0;
          for (int j = 0; j < 3; ++j) {
            int f[3] = {j == 0, j == 1, j == 2};
            for (int s2 = -1; s2 <= 1; s2 += 2) {
              if (s2 == 1 && j == i) {
                int l3 = lay_of(w, K[0] + f[0], K[1] + f[1], K[2] + f[2], &v3);
                if (v3 && l3 < lay) { ++n; val += rd_u(w, fld, j, K, f[0], f[1], f[2]); }
              } else if (s2 == -1 && j == i) {
              } else {
                int d4[3] = {s2 * f[0], s2 * f[1], s2 * f[2]};
                int l4 = lay_of(w, K[0] + d4[0], K[1] + d4[1], K[2] + d4[2], &v4);
                if (v4) {
                  int d3[3] = {d4[0] - e[0], d4[1] - e[1], d4[2] - e[2]};
                  int l3 = lay_of(w, K[0] + d3[0], K[1] + d3[1], K[2] + d3[2], &v3);
                  if (v3 && (l3 < lay || l4 < lay)) { ++n; val += rd_u(w, fld, i, K, d4[0], d4[1], d4[2]); }
                }
              }
            }
          }
          set_u(B(c), B(c)->u[fld][i], c.o, i, val / n, 0);
        }
      }
    }
    keylist t = set; set = set2; set2 = t; set2.n = 0;
    ++lay;
    if (set.n == 0) break;
  }
  free(set.k); free(set2.k);
}

static void alg_extrapolate(world_t* w) { alg_extrapolate_f(w, 0); }

/* ------------------------------------------------------------- particles */
/* Speed read through grid[key] semantics: the interpolation's m_grid[key]
 * creates the base cell (src/Policy_Speed_Interpolation_Linear_Symmetric.h:115). */
static double interp_rec(world_t* w, const double* d, int i, const int k[3], int comp, int sym) {
  double w0, w1;
  if (sym && i == comp) { w0 = 0.5 - d[i]; w1 = 0.5 + d[i]; }
  else { w0 = 1 - d[i]; w1 = d[i]; }
  int k1[3] = {k[0] + (i == 0), k[1] + (i == 1), k[2] + (i == 2)};
  if (i < 2) return w0 * interp_rec(w, d, i + 1, k, comp, sym) + w1 * interp_rec(w, d, i + 1, k1, comp, sym);
  return w0 * rd_u(w, w->ispeed, comp, k, 0, 0, 0) + w1 * rd_u(w, w->ispeed, comp, k1, 0, 0, 0);
}

/* Get_Speed of Policy_Speed_Interpolation_Linear_Symmetric
 * (src/Policy_Speed_Interpolation_Linear_Symmetric.h:79-119) when sym != 0,
 * of Policy_Speed_Interpolation_Linear (src/Policy_Speed_Interpolation_Linear.h:64-106)
 * otherwise. */
static void get_speed(world_t* w, const double pos[3], double out[3], int sym) {
  double pd[3];
  int k0[3];
  for (int i = 0; i < 3; ++i) {
    pd[i] = pos[i] * w->ih[i];
    k0[i] = (int)lround(pd[i]);
    pd[i] -= k0[i];
  }
  for (int k = 0; k < 3; ++k) {
    if (!sym) pd[k] += 0.5;
    int key[3];
    double d2[3];
    for (int j = 0; j < 3; ++j) {
      if (j != k && pd[j] < 0) { key[j] = k0[j] - 1; d2[j] = 1 + pd[j]; }
      else { key[j] = k0[j]; d2[j] = pd[j]; }
    }
    cell_get(w, key[0], key[1], key[2]);
    out[k] = interp_rec(w, d2, 0, key, k, sym);
    if (!sym) pd[k] -= 0.5;
  }
}

/* Algorithms_Move_Particles::Do (src/Algorithms_Move_Particles.h:29-32) with
 * Policy_Advance_Ode_RungeKutta::AdvanceSolveODE (src/Policy_Advance_ODE_RungeKutta.h:15-27). */
static void alg_move(world_t* w, int sym) {
  double dt = w->hdr.dt;
  for (int64_t q = 0; q < w->np; ++q) {
    double* pos = w->pos + 3 * q;
    double res[3], k[3], a[3], v[3];
    for (int i = 0; i < 3; ++i) res[i] = pos[i];
    get_speed(w, pos, v, sym);
    for (int i = 0; i < 3; ++i) { k[i] = dt * v[i]; res[i] += (1. / 6.) * k[i]; }
    for (int i = 0; i < 3; ++i) a[i] = pos[i] + k[i] * 0.5;
    get_speed(w, a, v, sym);
    for (int i = 0; i < 3; ++i) { k[i] = dt * v[i]; res[i] += (1. / 3.) * k[i]; }
    for (int i = 0; i < 3; ++i) a[i] = pos[i] + k[i] * 0.5;
    get_speed(w, a, v, sym);
    for (int i = 0; i < 3; ++i) { k[i] = dt * v[i]; res[i] += (1. / 3.) * k[i]; }
    for (int i = 0; i < 3; ++i) a[i] = pos[i] + k[i];
    get_speed(w, a, v, sym);
    for (int i = 0; i < 3; ++i) { k[i] = dt * v[i]; res[i] += (1. / 6.) * k[i]; }
    for (int i = 0; i < 3; ++i) pos[i] = res[i];
  }
}

/* ---------------------------------------------------------- setup passes */
/* src/Algorithms_Solid_To_Const.h:32-58 */
/* ------------------------------------------- boundary-condition extrapolation
 * Algorithm_Extrapolate_Boundary_Condition, 3D form
 * (src/Algorithm_Extrapolate_Boundary_Condition.h:454-975, common part :52-252)
 * with Policy_Is_In_Domain_Speed (src/Policy_Is_In_Domain_Speed.h:15-48), on
 * speed buffer w->ispeed, every write through the non-forced Set (const faces
 * keep their value).
 *
 * Visiting order. The reference visits its hash map's order, and a boundary
 * cell's case writes faces that later cells read, so its result depends on
 * that order. Here the order is fixed: cells by colour (x mod 5, y mod 5,
 * z mod 5), colours in turn, keys in order within a colour; the stack of
 * three-face corners is unwound in the reverse order (LIFO, :489-494). Every
 * read and write of one cell's case lies within Chebyshev distance 2 of the
 * cell, so two cells of one colour (5 or more apart on some axis) never touch
 * the same face and a colour's cells commute: the device runs each colour in
 * parallel and reaches the same values.
 *
 * Reference details kept: GetNeighbour(i, 0) is the -e_i neighbour (so
 * apply_nan_extrap counts it twice), Apply_Div_3d keeps only the last
 * tangential term, the n == 1 case's flag b is never cleared. An air or
 * missing neighbour counts as "not a boundary" where the reference reads an
 * unset counter; a read of a missing cell gives NaN (the reference would
 * dereference a null chunk), a write to one is dropped. The 3x3 corner
 * systems, which the reference hands to its Umfpack policy, are solved by
 * Gaussian elimination with partial pivoting (mac_solve3, solve3.h; the device
 * repeats its operations). */
static int eb_valid(world_t* w, int x, int y, int z) { return cell_valid(w, cell_at(w, x, y, z)); }
static int eb_air(world_t* w, int x, int y, int z) {
  cell_t c = cell_at(w, x, y, z);
  return !cell_valid(w, c) || is_air(B(c)->type[c.o]);
}
static double eb_u(world_t* w, const int k[3], int i) { /* i: 1..3 */
  cell_t c = cell_at(w, k[0], k[1], k[2]);
  return cell_valid(w, c) ? B(c)->u[w->ispeed][i - 1][c.o] : NAN;
}
static void eb_set(world_t* w, const int k[3], int i, double v) {
  cell_t c = cell_at(w, k[0], k[1], k[2]);
  if (cell_valid(w, c)) set_u(B(c), B(c)->u[w->ispeed][i - 1], c.o, i - 1, v, 0);
}
/* key + s e_i (i 1..3; s = 0 means -1, as the neighbour tables index (s + 1) >> 1) */
static void eb_nb(const int k[3], int i, int s, int out[3]) {
  out[0] = k[0]; out[1] = k[1]; out[2] = k[2];
  out[i - 1] += s > 0 ? 1 : -1;
}
/* IsBoundary (:89-119): the air face-neighbours in (i, s) order; 0 for an air
 * or missing cell */
static int eb_boundary(world_t* w, const int k[3], int dir[6], int sign[6]) {
  if (!eb_valid(w, k[0], k[1], k[2]) || eb_air(w, k[0], k[1], k[2])) return 0;
  int n = 0;
  for (int i = 1; i <= 3; ++i)
    for (int s = -1; s <= 1; s += 2) {
      int k2[3];
      eb_nb(k, i, s, k2);
      if (eb_valid(w, k2[0], k2[1], k2[2]) && eb_air(w, k2[0], k2[1], k2[2])) {
        dir[n] = i;
        sign[n] = s;
        ++n;
      }
    }
  return n;
}
static void eb_set_nan(world_t* w, const int k[3]) { /* apply_set_nan (:149-177) */
  if (eb_air(w, k[0], k[1], k[2]) == 0) return;
  for (int i = 1; i <= 3; ++i)
    for (int s = -1; s <= 1; s += 2) {
      int k2[3];
      eb_nb(k, i, s, k2);
      if (eb_valid(w, k2[0], k2[1], k2[2])) {
        if (eb_air(w, k2[0], k2[1], k2[2])) eb_set(w, s == -1 ? k : k2, i, NAN);
      } else if (s == -1) {
        eb_set(w, k, i, NAN);
      }
    }
}
static int eb_in_domain(world_t* w, const int k[3], int d) { /* Get_Is_Speed_In_Domain */
  int k2[3], k3[3];
  eb_nb(k, d, -1, k2);
  const int f1 = !eb_air(w, k[0], k[1], k[2]);
  if (!eb_valid(w, k2[0], k2[1], k2[2])) return f1;
  const int f2 = !eb_air(w, k2[0], k2[1], k2[2]);
  if (f1 && f2) return 1;
  if (!f1 && !f2) return 0;
  if (f1) eb_nb(k, d, 1, k3);
  else eb_nb(k2, d, -1, k3);
  if (!eb_valid(w, k3[0], k3[1], k3[2])) return 1;
  return eb_air(w, k3[0], k3[1], k3[2]);
}
static void eb_div(world_t* w, const int k[3], int d, int sign) { /* Apply_Div_3d (:912-932) */
  int n[3];
  eb_nb(k, d, 1, n);
  double v = eb_u(w, k, d);
  if (sign == -1) {
    v = eb_u(w, n, d);
    n[0] = k[0]; n[1] = k[1]; n[2] = k[2];
  }
  double res = 0;
  for (int d2 = 1; d2 <= 3; ++d2) {
    if (d2 == d) continue;
    int k3[3];
    eb_nb(k, d2, 1, k3);
    res = w->ih[d2 - 1] * (eb_u(w, k3, d2) - eb_u(w, k, d2));
  }
  res = v - sign * res * w->h[d - 1];
  eb_set(w, n, d, res);
}
static void eb_plane(world_t* w, const int a[3], const int b[3], int d, int sign, int d2) { /* Apply_3d_Plane (:897-911) */
  int n[3] = {a[0], a[1], a[2]}, n2[3] = {b[0], b[1], b[2]};
  if (sign == 1) {
    eb_nb(a, d, 1, n);
    eb_nb(b, d, 1, n2);
  }
  const double v1 = eb_u(w, n, d), v2 = eb_u(w, n2, d), v3 = eb_u(w, b, d2);
  const double v = -sign * w->ih[d2 - 1] * w->h[d - 1] * (v2 - v1) + v3;
  int k3[3];
  eb_nb(b, d, sign, k3);
  eb_set(w, k3, d2, v);
}
static void eb_plane45(world_t* w, const int k[3], int sa, int da, int sb, int db) { /* Apply_3d_Plane_45 (:934-952) */
  int n1[3], n2[3];
  eb_nb(k, da, 1, n1);
  eb_nb(k, db, 1, n2);
  double v1 = eb_u(w, k, da), v2 = eb_u(w, k, db);
  if (sa == -1) {
    v1 = eb_u(w, n1, da);
    n1[0] = k[0]; n1[1] = k[1]; n1[2] = k[2];
  }
  if (sb == -1) {
    v2 = eb_u(w, n2, db);
    n2[0] = k[0]; n2[1] = k[1]; n2[2] = k[2];
  }
  eb_set(w, n1, da, v1);
  eb_set(w, n2, db, v2);
}
/* Choose_Boundary_Case_3d (:793-890) for all but the n == 3 corners, which
 * the caller keeps for eb_corner. */
static void eb_choose(world_t* w, const int k[3], const int* dir, const int* sign, int n) {
  if (n == 1) {
    eb_div(w, k, dir[0], sign[0]);
    for (int d2 = 1; d2 <= 3; ++d2) {
      if (d2 == dir[0]) continue;
      for (int i = -1; i <= 1; i += 2) {
        int k2[3], dt[6], st[6];
        eb_nb(k, d2, i, k2);
        const int nt = eb_boundary(w, k2, dt, st);
        if (nt == 1) eb_div(w, k2, dt[0], st[0]);
        if (nt == 1 && dt[0] == dir[0]) {
          if (i < 0) eb_plane(w, k2, k, dir[0], sign[0], d2);
          else eb_plane(w, k, k2, dir[0], sign[0], d2);
        }
      }
      int k3[3] = {k[0], k[1], k[2]};
      if (sign[0] == 1) eb_nb(k, dir[0], 1, k3);
      if (!eb_in_domain(w, k, dir[0])) eb_set(w, k3, dir[0], NAN);
    }
  } else if (n == 2) {
    if (dir[0] != dir[1]) eb_plane45(w, k, sign[0], dir[0], sign[1], dir[1]);
  } else if (n != 3) {
    for (int i = 0; i < n; ++i) {
      int k2[3] = {k[0], k[1], k[2]};
      if (sign[i] == 1) eb_nb(k, dir[i], 1, k2);
      if (!eb_in_domain(w, k2, dir[i])) eb_set(w, k2, dir[i], NAN);
    }
  }
}
/* The n == 3 corner signs (s1, s2, s3) or 0 when an axis repeats. */
static int eb_corner_signs(const int* dir, const int* sign, int n, int s[3]) {
  s[0] = s[1] = s[2] = 0;
  for (int a = 1; a <= 3; ++a)
    for (int i = 0; i < n; ++i)
      if (dir[i] == a) {
        s[a - 1] = sign[i];
        break;
      }
  return s[0] != 0 && s[1] != 0 && s[2] != 0;
}
/* SolveMatrix (:571-775): the 3x3 system of CreateMatrix (:551-570; its CSC
 * value[3 j + r] is A[r][j], so A below is row-major) with the right-hand
 * side of the reference's terms, in their order. */
static void eb_corner(world_t* w, const int k[3], int s1, int s2, int s3) {
  const double* ih = w->ih;
  const double A[9] = {
      -s1 * 2 * ih[0] - s1 * 0.5 * ih[2], s2 * 2 * ih[1] + s2 * 0.5 * ih[2], -s3 * 0.5 * ih[0] + s2 * s3 * 0.5 * ih[1],
      -s1 * 0.5 * ih[2] + s1 * 0.5 * ih[1], s2 * 2 * ih[1] + s2 * 0.5 * ih[1], -s3 * 2 * ih[2] - s3 * 0.5 * ih[0],
      s1 * ih[0], s2 * ih[1], s3 * ih[2]};
  int e1[3], e2[3], e3[3], m1[3], m2[3], m3[3], t[3];
  eb_nb(k, 1, 1, e1);
  eb_nb(k, 2, 1, e2);
  eb_nb(k, 3, 1, e3);
  eb_nb(k, 1, -s1, m1);
  eb_nb(k, 2, -s2, m2);
  eb_nb(k, 3, -s3, m3);
#define U(key, i) eb_u(w, key, i)
  double b[3], x[3];
  b[0] = 0;
  b[0] += s1 == 1 ? -2 * ih[0] * U(k, 1) : 2 * ih[0] * U(e1, 1);
  b[0] += s2 == 1 ? 2 * ih[1] * U(k, 2) : -2 * ih[1] * U(e2, 2);
  b[0] += s3 == 1 ? 0.5 * ih[0] * U(k, 3) : -0.5 * ih[0] * U(e3, 3);
  eb_nb(m1, 3, 1, t);
  b[0] += s3 * 0.5 * ih[0] * (-U(m1, 3) - U(t, 3));
  b[0] += s1 == 1 ? 0.5 * ih[2] * U(k, 1) : -0.5 * ih[2] * U(e1, 1);
  eb_nb(m3, 1, 1, t);
  b[0] += s1 * 0.5 * ih[2] * (-U(m3, 1) - U(t, 1));
  b[0] += s3 == 1 ? -0.5 * ih[1] * U(k, 3) : 0.5 * ih[1] * U(e3, 3);
  eb_nb(m2, 3, 1, t);
  b[0] += s3 * 0.5 * ih[1] * (U(m2, 3) + U(t, 3));
  b[0] += s2 == 1 ? -0.5 * ih[2] * U(k, 2) : 0.5 * ih[2] * U(e2, 2);
  eb_nb(m3, 2, 1, t);
  b[0] += s2 * 0.5 * ih[2] * (U(m3, 2) + U(t, 2));
  b[1] = 0;
  b[1] += s3 == 1 ? -2 * ih[2] * U(k, 3) : 2 * ih[2] * U(m3, 3);
  b[1] += s2 == 1 ? 2 * ih[1] * U(k, 2) : -2 * ih[1] * U(e2, 2);
  b[1] += s3 == 1 ? 0.5 * ih[0] * U(k, 3) : -0.5 * ih[0] * U(e3, 3);
  eb_nb(m1, 3, 1, t);
  b[1] += s3 * 0.5 * ih[0] * (-U(m1, 3) - U(t, 3));
  b[1] += s1 == 1 ? 0.5 * ih[2] * U(k, 1) : -0.5 * ih[2] * U(e1, 1);
  eb_nb(m3, 1, 1, t);
  b[1] += s1 * 0.5 * ih[2] * (-U(m3, 1) - U(t, 1));
  b[1] += s1 == 1 ? -0.5 * ih[1] * U(k, 1) : -0.5 * ih[1] * U(e1, 1);
  eb_nb(m2, 1, 1, t);
  b[1] += s1 * 0.5 * ih[1] * (U(m2, 1) + U(t, 1));
  b[1] += s2 == 1 ? -0.5 * ih[0] * U(k, 2) : 0.5 * ih[0] * U(e2, 2);
  eb_nb(m1, 2, 1, t);
  b[1] += s2 * 0.5 * ih[0] * (U(m1, 2) + U(t, 2));
  b[2] = 0;
  b[2] += s1 == 1 ? ih[0] * U(k, 1) : -ih[0] * U(e1, 1);
  b[2] += s2 == 1 ? ih[1] * U(k, 2) : -ih[1] * U(e2, 2);
  b[2] += s3 == 1 ? ih[2] * U(k, 3) : -ih[2] * U(e3, 3);
#undef U
  if (!isnan(b[0]) && !isnan(b[1]) && !isnan(b[2])) {
    mac_solve3(A, b, x);
  } else {
    x[0] = x[1] = x[2] = NAN;
  }
  eb_set(w, s1 == 1 ? e1 : k, 1, x[0]);
  eb_set(w, s2 == 1 ? e2 : k, 2, x[1]);
  eb_set(w, s3 == 1 ? e3 : k, 3, x[2]);
}
/* apply_nan_extrap (:183-251) */
static void eb_nan_extrap(world_t* w, const int k[3]) {
  int tab[2][6], n = 0;
  for (int i = 1; i <= 3; ++i) {
    int e[3];
    eb_nb(k, i, 1, e);
    if (isnan(eb_u(w, k, i))) { tab[0][n] = i; tab[1][n] = 0; ++n; }
    if (isnan(eb_u(w, e, i))) { tab[0][n] = i; tab[1][n] = 1; ++n; }
  }
  if (n == 0) return;
  for (int j = 0; j < n; ++j) {
    const int d = tab[0][j];
    int k2[3] = {k[0], k[1], k[2]};
    if (tab[1][j] == 1) eb_nb(k, d, 1, k2);
    double vt = 0;
    int nb = 0;
    for (int d2 = 1; d2 <= 3; ++d2)
      for (int s = -1; s <= 1; ++s) {
        int k3[3];
        eb_nb(k2, d2, s, k3);
        const double add = eb_u(w, k3, d);
        if (!isnan(add)) {
          vt += add;
          ++nb;
        }
      }
    if (nb != 0) vt /= nb;
    eb_set(w, k2, d, vt);
  }
  double div = 0;
  for (int i = 1; i <= 3; ++i) {
    int e[3];
    eb_nb(k, i, 1, e);
    div += w->ih[i - 1] * (eb_u(w, e, i) - eb_u(w, k, i));
  }
  const double cor = div / n;
  for (int j = 0; j < n; ++j) {
    const int d = tab[0][j], sg = tab[1][j];
    int k2[3] = {k[0], k[1], k[2]};
    if (sg == 1) eb_nb(k, d, 1, k2);
    eb_set(w, k2, d, eb_u(w, k2, d) - (2 * sg - 1) * w->h[d - 1] * cor);
  }
}
static int eb_mod5(int v) { return ((v % 5) + 5) % 5; }
static int eb_color(const int* k) { return eb_mod5(k[0]) + 5 * eb_mod5(k[1]) + 25 * eb_mod5(k[2]); }
static int cmp_color_key(const void* a, const void* b) {
  const int* x = (const int*)a;
  const int* y = (const int*)b;
  const int cx = eb_color(x), cy = eb_color(y);
  if (cx != cy) return cx < cy ? -1 : 1;
  for (int i = 2; i >= 0; --i)
    if (x[i] != y[i]) return x[i] < y[i] ? -1 : 1;
  return 0;
}
static int cmp_color_key_rev(const void* a, const void* b) {
  const int cx = eb_color((const int*)a), cy = eb_color((const int*)b);
  if (cx != cy) return cx < cy ? -1 : 1;
  return -cmp_color_key(a, b);
}
static int cmp_key_zyx(const void* a, const void* b) {
  const int* x = (const int*)a;
  const int* y = (const int*)b;
  for (int i = 2; i >= 0; --i)
    if (x[i] != y[i]) return x[i] < y[i] ? -1 : 1;
  return 0;
}
/* order 0: colour-major, keys ascending within a colour (the device's order);
 * 1: key order (z, then y, then x), within one chunk the reference's own order
 * (offsets x + 8y + 64z), which the tests use to compare with the reference
 * run on single-chunk worlds; 2: colour-major, keys descending within a
 * colour (the tests check that it changes nothing). */
static void alg_extrap_bc(world_t* w, int order) {
  /* the existing cells in colour-major order */
  int64_t n = 0;
  for (int64_t bi = 0; bi < w->nb; ++bi)
    for (int o = 0; o < 512; ++o) n += w->b[bi]->exists[o] != 0;
  int* keys = (int*)malloc(sizeof(int) * 3 * (size_t)(n ? n : 1));
  int64_t m = 0;
  for (int64_t bi = 0; bi < w->nb; ++bi)
    for (int o = 0; o < 512; ++o)
      if (w->b[bi]->exists[o]) key_of(w, bi, o, keys + 3 * m++);
  qsort(keys, (size_t)n, 3 * sizeof(int), order == 1 ? cmp_key_zyx : (order == 2 ? cmp_color_key_rev : cmp_color_key));
  for (int64_t i = 0; i < n; ++i) eb_set_nan(w, keys + 3 * i);
  int* corners = (int*)malloc(sizeof(int) * 6 * (size_t)(n ? n : 1));
  int64_t nc = 0;
  for (int64_t i = 0; i < n; ++i) {
    int dir[6], sign[6], s[3];
    const int nn = eb_boundary(w, keys + 3 * i, dir, sign);
    if (nn == 0) continue;
    if (nn == 3) {
      if (eb_corner_signs(dir, sign, nn, s)) {
        memcpy(corners + 6 * nc, keys + 3 * i, 3 * sizeof(int));
        memcpy(corners + 6 * nc + 3, s, 3 * sizeof(int));
        ++nc;
      }
      continue;
    }
    eb_choose(w, keys + 3 * i, dir, sign, nn);
  }
  for (int64_t i = nc - 1; i >= 0; --i)
    eb_corner(w, corners + 6 * i, corners[6 * i + 3], corners[6 * i + 4], corners[6 * i + 5]);
  for (int64_t i = 0; i < n; ++i) {
    int dir[6], sign[6];
    if (eb_boundary(w, keys + 3 * i, dir, sign)) eb_nan_extrap(w, keys + 3 * i);
  }
  free(corners);
  free(keys);
}

static void alg_solid_to_const(world_t* w) {
  keylist s = {0};
  for (int64_t bi = 0; bi < w->nb; ++bi)
    for (int o = 0; o < 512; ++o)
      if (w->b[bi]->exists[o] && w->b[bi]->type[o] == MAC_SOLID) {
        int k[3];
        key_of(w, bi, o, k);
        kl_push(&s, k);
      }
  for (int64_t q = s.n - 1; q >= 0; --q) {
    int* k = s.k + 3 * q;
    cell_t c = cell_get(w, k[0], k[1], k[2]);
    B(c)->flags[c.o] |= MAC_FLAG_NODELETE;
    B(c)->p[c.o] = 0;
    for (int i = 0; i < 3; ++i) {
      c = cell_get(w, k[0], k[1], k[2]);
      set_u(B(c), B(c)->u[0][i], c.o, i, 0.0, 0);
      B(c)->flags[c.o] |= (uint8_t)(1u << i);
      cell_t n = cell_get(w, k[0] + (i == 0), k[1] + (i == 1), k[2] + (i == 2));
      B(n)->flags[n.o] |= MAC_FLAG_NODELETE;
      for (int j = 0; j < 3; ++j) set_u(B(n), B(n)->u[0][j], n.o, j, 0.0, 0);
      B(n)->p[n.o] = 0;
      B(n)->flags[n.o] |= (uint8_t)(1u << i);
    }
  }
  free(s.k);
}

/* src/Algorithms_Speed_Constant_Mirror.h:22-70 */
static void alg_mirror(world_t* w) {
  keylist s = {0};
  for (int64_t bi = 0; bi < w->nb; ++bi)
    for (int o = 0; o < 512; ++o)
      if (w->b[bi]->exists[o] && (w->b[bi]->flags[o] & 7)) {
        int k[3];
        key_of(w, bi, o, k);
        kl_push(&s, k);
      }
  for (int64_t q = 0; q < s.n; ++q) {
    int* k = s.k + 3 * q;
    for (int i = 0; i < 3; ++i) {
      cell_t n = cell_get(w, k[0] + (i == 0), k[1] + (i == 1), k[2] + (i == 2));
      for (int j = 0; j < 3; ++j) set_u(B(n), B(n)->u[0][j], n.o, j, 0.0, 0);
    }
  }
  for (int64_t q = 0; q < s.n; ++q) {
    int* k = s.k + 3 * q;
    for (int i = 0; i < 3; ++i) {
      cell_t n = cell_get(w, k[0] + (i == 0), k[1] + (i == 1), k[2] + (i == 2));
      cell_t c = cell_get(w, k[0], k[1], k[2]);
      if ((B(c)->flags[c.o] >> i) & 1) set_u(B(n), B(n)->u[0][i], n.o, i, B(c)->u[0][i][c.o], 0);
    }
  }
  free(s.k);
}

/* ------------------------------------------------------------ pipeline B */
/* src/Algorithms_Create_Interior_Depth.h:20-40: the stage form of the refill
 * (no particles): inflow cells still empty get layer 0 and SetFluid, interior
 * cells get layer 0. */
static void alg_create_interior_depth(world_t* w) {
  for (int64_t bi = 0; bi < w->nb; ++bi) {
    brick_t* b = w->b[bi];
    for (int o = 0; o < 512; ++o) {
      if (!b->exists[o]) continue;
      if (b->type[o] == MAC_INFLOW && b->layer[o] == -1) {
        b->layer[o] = 0;
        b->type[o] = set_fluid(b->type[o]);
      } else if (b->type[o] == MAC_INTERIOR) {
        b->layer[o] = 0;
      }
    }
  }
}

/* One stage's Policy::Do() of test/Jet3.cpp:642-675: Algorithms<solve_grid,
 * force projection, extrapolation of the acceleration>, where solve_grid =
 * Algorithms<init2, Gravity, Convection, Viscosity> and init2 the depth
 * topology with Create_Interior_Depth and Algorithms_Extrapolate (the
 * boundary-condition extrapolation is not composed). The force projection
 * (src/Algorithms_Solve_Pressure_Force.h:16-24) assembles, projects the
 * acceleration with Dirichlet pressures from the current speed buffer, and
 * Algorithms_Accel_To_Speed (src/Algorithms_Accel_To_Speed.h:26-31) runs the
 * extrapolation on the acceleration. */
static void stage_solve_grid_force(world_t* w) {
  alg_initialize_depth(w);
  alg_layer_initial_depth(w);
  alg_create_interior_depth(w);
  alg_update_layer_depth(w);
  alg_delete(w);
  alg_extrapolate_f(w, w->ispeed);
  grid_forces(w, w->ispeed);
  csr_t A;
  assemble(w, &A);
  project_field(w, &A, ACC, w->ispeed);
  csr_free(&A);
  alg_extrapolate_f(w, ACC);
}

/* Algorithms_RungeKutta_all::Do (src/Algorithms_RungeKutta_all.h:35-156) with
 * Policy_Move_Particle (src/Policy_Move_Particle.h:24-56): four stages over
 * speed buffers 0..2 and particle positions 0..2 in the reference's order
 * (the grid update of a stage comes before its particle update, which reads
 * the updated speed; the stage-2/3 update of position 1 reads the speed at the
 * position 2 just written). Forced sets except the final speed. */
static void alg_rk_all(world_t* w) {
  const double dt = w->hdr.dt;
  const int sym = w->hdr.interp_symmetric != 0;
  w->ispeed = 0;
  w->imove = 0;
  acc_zero(w);
  for (int stage = 1; stage <= 4; ++stage) {
    stage_solve_grid_force(w);
    for (int64_t bi = 0; bi < w->nb; ++bi) {
      brick_t* b = w->b[bi];
      for (int o = 0; o < 512; ++o) {
        if (!b->exists[o]) continue;
        for (int i = 0; i < 3; ++i) {
          const double a = b->u[ACC][i][o];
          if (stage == 1) {
            b->u[2][i][o] = b->u[0][i][o] + a * dt * 0.5;
            b->u[1][i][o] = b->u[0][i][o] + a * dt * 1. / 6.;
          } else if (stage == 2) {
            b->u[2][i][o] = b->u[0][i][o] + a * dt * 0.5;
            b->u[1][i][o] = b->u[1][i][o] + a * dt * 1. / 3.;
          } else if (stage == 3) {
            b->u[2][i][o] = b->u[0][i][o] + a * dt;
            b->u[1][i][o] = b->u[1][i][o] + a * dt * 1. / 3.;
          } else {
            set_u(b, b->u[0][i], o, i, b->u[1][i][o] + a * dt * 1. / 6., 0);
          }
        }
      }
    }
    for (int64_t q = 0; q < w->np; ++q) {
      double* p0 = pbuf(w, 0, q);
      double* p1 = pbuf(w, 1, q);
      double* p2 = pbuf(w, 2, q);
      double v[3];
      if (stage == 1) {
        get_speed(w, p0, v, sym);
        for (int i = 0; i < 3; ++i) p2[i] = p0[i] + dt * 0.5 * v[i];
        get_speed(w, p0, v, sym);
        for (int i = 0; i < 3; ++i) p1[i] = p0[i] + dt * 1.0 / 6.0 * v[i];
      } else if (stage == 2 || stage == 3) {
        const double s2 = stage == 2 ? dt * 0.5 : dt;
        get_speed(w, p2, v, sym);
        for (int i = 0; i < 3; ++i) p2[i] = p0[i] + s2 * v[i];
        get_speed(w, p2, v, sym);
        for (int i = 0; i < 3; ++i) p1[i] = p1[i] + dt * 1.0 / 3.0 * v[i];
      } else {
        get_speed(w, p2, v, sym);
        for (int i = 0; i < 3; ++i) p0[i] = p1[i] + dt * 1.0 / 6.0 * v[i];
      }
    }
    if (stage < 4) acc_zero(w);
    if (stage == 1) {
      w->hdr.t += 0.5 * dt;
      w->ispeed = 2;
      w->imove = 2;
    } else if (stage == 3) {
      w->hdr.t += 0.5 * dt;
    }
  }
  w->ispeed = 0;
  w->imove = 0;
}

/* The per-step init of pipeline B (test/Jet3.cpp:546 without the jet's own
 * particle filter and the boundary-condition extrapolation): the depth
 * topology with the refill, dt, and Algorithms_Extrapolate on speed 0. */
static void alg_init_b(world_t* w) {
  alg_initialize_depth(w);
  alg_layer_initial_depth(w);
  alg_create_fluid_depth(w);
  alg_update_layer_depth(w);
  alg_delete(w);
  alg_dt(w);
  alg_extrapolate_f(w, 0);
}

/* --------------------------------------------------------------- driver */
static world_t* world_from_file(const mac_state_file* st) {
  world_t* w = (world_t*)calloc(1, sizeof(world_t));
  w->hdr = st->hdr;
  for (int i = 0; i < 3; ++i) { w->h[i] = st->hdr.h[i]; w->ih[i] = 1 / st->hdr.h[i]; }
  w->seed = st->hdr.step;
  hash_rebuild(w);
  for (int64_t c = 0; c < st->hdr.nchunks; ++c) {
    int64_t bi = brick_create(w, st->keys[3 * c], st->keys[3 * c + 1], st->keys[3 * c + 2]);
    brick_t* b = w->b[bi];
    size_t base = (size_t)c * 512;
    memcpy(b->exists, st->exists + base, 512);
    for (int k = 0; k < 2; ++k)
      for (int i = 0; i < 3; ++i) memcpy(b->u[k][i], st->u[k][i] + base, 512 * 8);
    for (int i = 0; i < 3; ++i) memcpy(b->u[ACC][i], st->acc[i] + base, 512 * 8);
    memcpy(b->p, st->p + base, 512 * 8);
    memcpy(b->flags, st->flags + base, 512);
    memcpy(b->type, st->type + base, 512);
    memcpy(b->layer, st->layer + base, 512 * 4);
    memcpy(b->id, st->id + base, 512 * 4);
    memcpy(b->depth, st->depth + base, 512 * 4);
  }
  for (int64_t q = 0; q < st->hdr.nparticles; ++q) add_particle(w, st->pos + 3 * q);
  return w;
}

static int cmp_keys(const void* a, const void* b) {
  const brick_t* x = *(brick_t* const*)a;
  const brick_t* y = *(brick_t* const*)b;
  for (int i = 2; i >= 0; --i)
    if (x->key[i] != y->key[i]) return x->key[i] < y->key[i] ? -1 : 1;
  return 0;
}

static void world_to_file(world_t* w, mac_state_file* st) {
  qsort(w->b, (size_t)w->nb, sizeof(brick_t*), cmp_keys);
  hash_rebuild(w);
  mac_state_alloc(st, w->nb, w->np);
  st->hdr = w->hdr;
  st->hdr.nchunks = w->nb;
  st->hdr.nparticles = w->np;
  st->hdr.step = w->seed;
  for (int64_t c = 0; c < w->nb; ++c) {
    brick_t* b = w->b[c];
    size_t base = (size_t)c * 512;
    memcpy(st->keys + 3 * c, b->key, 12);
    memcpy(st->exists + base, b->exists, 512);
    for (int k = 0; k < 2; ++k)
      for (int i = 0; i < 3; ++i) memcpy(st->u[k][i] + base, b->u[k][i], 512 * 8);
    for (int i = 0; i < 3; ++i) memcpy(st->acc[i] + base, b->u[ACC][i], 512 * 8);
    memcpy(st->p + base, b->p, 512 * 8);
    memcpy(st->flags + base, b->flags, 512);
    memcpy(st->type + base, b->type, 512);
    memcpy(st->layer + base, b->layer, 512 * 4);
    memcpy(st->id + base, b->id, 512 * 4);
    memcpy(st->depth + base, b->depth, 512 * 4);
  }
  memcpy(st->pos, w->pos, (size_t)w->np * 24);
}

static void world_free(world_t* w) {
  for (int64_t i = 0; i < w->nb; ++i) free(w->b[i]);
  free(w->b); free(w->hkeys); free(w->hval); free(w->pos); free(w->pos1); free(w->pos2); free(w);
}

static int64_t fluid_count(world_t* w) {
  int64_t n = 0;
  for (int64_t bi = 0; bi < w->nb; ++bi)
    for (int o = 0; o < 512; ++o) n += w->b[bi]->exists[o] && is_fluid(w->b[bi]->type[o]);
  return n;
}

static void topology(world_t* w) {
  if (w->hdr.depth_mode) {
    /* Algorithms<Initialize_Layer_And_Depth, Layer_Initial_With_Particle_Depth,
     * Create_Fluid_Particle_Depth, Update_CellType_Layer_Depth, Delete_MacCell,
     * Calculate_Time_Step> (test/Jet3.cpp:546, without the jet's own particle
     * filter and the extrapolations, which the step runs after the ODE) */
    alg_initialize_depth(w);
    alg_layer_initial_depth(w);
    alg_create_fluid_depth(w);
    alg_update_layer_depth(w);
  } else {
    alg_initialize(w);
    alg_layer_initial(w);
    alg_create_fluid(w);
    alg_update_layer(w);
  }
  alg_delete(w);
  alg_dt(w);
}

/* One named stage (same names as oracle/_ref/mac_ref) n times. Returns 0 on
 * success; stats[] receives invalid reads, created cells, CG iterations, the
 * last relative residual, the max |div| after the last projection and the
 * accumulated fluid cell-steps. */
int mac_oracle_run(const char* in_path, const char* out_path, const char* cmd, int n, double rtol,
                   double* stats) {
  mac_state_file st;
  if (mac_state_read(in_path, &st) != 0) return -1;
  world_t* w = world_from_file(&st);
  mac_state_free(&st);
  if (rtol > 0) g_rtol = rtol;
  int64_t fcs = 0;
  int sym = w->hdr.interp_symmetric != 0;
  for (int r = 0; r < n; ++r) {
    if (!strcmp(cmd, "firstinit")) {
      alg_solid_to_const(w);
      alg_mirror(w);
      if (w->hdr.depth_mode) {
        alg_initialize_depth(w);
        alg_create_fluid_depth(w);
        alg_layer_initial_depth(w);
        alg_update_layer_depth(w);
      } else {
        alg_initialize(w);
        alg_create_fluid(w);
        alg_layer_initial(w);
        alg_update_layer(w);
      }
      alg_delete(w);
      alg_extrapolate(w);
    } else if (!strcmp(cmd, "setup")) {
      alg_solid_to_const(w);
      alg_mirror(w);
    } else if (!strcmp(cmd, "step") || !strcmp(cmd, "bench")) {
      ++w->seed;
      topology(w);
      alg_rk2(w);
      alg_extrapolate(w);
      alg_move(w, sym);
      w->hdr.t += w->hdr.dt;
      fcs += fluid_count(w);
    } else if (!strcmp(cmd, "bstep")) {
      w->viscous = 1;
      ++w->seed;
      alg_init_b(w);
      alg_rk_all(w);
      fcs += fluid_count(w);
    } else if (!strcmp(cmd, "binit")) {
      w->viscous = 1;
      ++w->seed;
      alg_init_b(w);
    } else if (!strcmp(cmd, "bode")) {
      w->viscous = 1;
      alg_rk_all(w);
    } else if (!strcmp(cmd, "vstep")) {
      w->viscous = 1;
      ++w->seed;
      topology(w);
      alg_rk2(w);
      alg_extrapolate(w);
      alg_move(w, sym);
      w->hdr.t += w->hdr.dt;
      fcs += fluid_count(w);
    } else if (!strcmp(cmd, "vforces")) {
      w->viscous = 1;
      acc_zero(w);
      grid_forces(w, 0);
    } else if (!strcmp(cmd, "vode")) {
      w->viscous = 1;
      alg_rk2(w);
    } else if (!strcmp(cmd, "vproject")) {
      w->viscous = 1;
      alg_project(w);
    } else if (!strcmp(cmd, "topology")) {
      ++w->seed;
      topology(w);
    } else if (!strcmp(cmd, "forces")) {
      acc_zero(w);
      alg_gravity(w, 0);
      alg_convection(w, 0);
    } else if (!strcmp(cmd, "ode")) {
      alg_rk2(w);
    } else if (!strcmp(cmd, "project")) {
      alg_project(w);
    } else if (!strcmp(cmd, "extrapolate")) {
      alg_extrapolate(w);
    } else if (!strcmp(cmd, "extrapbc")) {
      alg_extrap_bc(w, 0);
    } else if (!strcmp(cmd, "extrapbckey")) {
      alg_extrap_bc(w, 1);
    } else if (!strcmp(cmd, "extrapbcrev")) {
      alg_extrap_bc(w, 2);
    } else if (!strcmp(cmd, "move")) {
      alg_move(w, 1);
    } else if (!strcmp(cmd, "movelin")) {
      alg_move(w, 0);
    } else {
      world_free(w);
      return -2;
    }
  }
  if (stats) {
    stats[0] = (double)w->invalid_reads;
    stats[1] = (double)w->created_cells;
    stats[2] = (double)w->cg_iters;
    stats[3] = w->last_relres;
    stats[4] = w->max_div;
    stats[5] = (double)fcs;
  }
  int rc = 0;
  if (out_path && out_path[0]) {
    world_to_file(w, &st);
    rc = mac_state_write(out_path, &st);
    mac_state_free(&st);
  }
  world_free(w);
  return rc;
}

/* Single-policy probes on a state (for the reference's known-answer tests):
 * what = 0: Get_Speed(pos) of the symmetric (sym != 0) or plain interpolation,
 *           out[0..2];
 * what = 1: Get_Convection_Speed(cell key, axis i) of the upwind policy, out[0];
 * what = 2: Get_Divergence(cell key), out[0];
 * what = 3: Get_Gradiant(cell key, axis i) from the stored pressures, out[0]. */
int mac_oracle_probe(const char* in_path, int what, const double* pos, const int* key, int i, int sym,
                     double* out) {
  mac_state_file st;
  if (mac_state_read(in_path, &st) != 0) return -1;
  world_t* w = world_from_file(&st);
  mac_state_free(&st);
  if (what == 0) {
    get_speed(w, pos, out, sym);
  } else if (what == 1) {
    out[0] = convection_speed(w, 0, key, i);
  } else if (what == 2) {
    out[0] = divergence(w, 0, key);
  } else if (what == 3) {
    cell_t c = cell_at(w, key[0], key[1], key[2]);
    double g = (c.b >= 0 ? B(c)->p[c.o] : 0.0) * w->ih[i];
    g -= rd_p(w, key, -(i == 0), -(i == 1), -(i == 2)) * w->ih[i];
    out[0] = g;
  } else {
    world_free(w);
    return -2;
  }
  world_free(w);
  return 0;
}

/* The jitter function, exported so the tests can compare it with the device's. */
void mac_oracle_jitter8(uint64_t seed, int kx, int ky, int kz, int s, double hx, double hy,
                        double hz, double* out) {
  mac_jitter8_position(seed, kx, ky, kz, s, hx, hy, hz, out);
}

/* The material rules, exported so the tests can check them against the
 * reference's own truth tables (test/TestData_CellType_Fluid_Air_Solid_Inflow*.h,
 * test/Test_Data_CellType_Domain_Fluid.h): out[0] GetIsFluid, out[1] GetIsAir,
 * out[2] GetIsInDomain, out[3] the material after SetAir, out[4] after SetFluid
 * (src/Data_CellType_Fluid_Air_Solid_Inflow_Interior.tpp:178-193). */
void mac_oracle_material(int code, int* out) {
  const uint8_t t = (uint8_t)code;
  out[0] = is_fluid(t);
  out[1] = is_air(t);
  out[2] = in_domain(t);
  out[3] = set_air(t);
  out[4] = set_fluid(t);
}
