/* State-file format shared by the oracle programs (test infrastructure only).
 *
 * A state is the full content of the reference's sparse chunk grid
 * (src/ChunkHashTable.h:22-160 with 8^3 chunks) plus its particle list
 * (src/TableContainerList.h:24-25) and timing (src/Data_Timing_Time.h:7-9).
 * Every one of the 512 cells of a live chunk is stored, including cells whose
 * existence bit is clear: the reference keeps their data and reuses it when
 * the cell is re-created by operator[] (src/ChunkHashTable.tpp:62-87).
 *
 * Little-endian layout:
 *   header (256 bytes, mac_state_header)
 *   int32  keys[nchunks][3]            chunk keys, sorted by (z, y, x)
 *   uint8  exists[nchunks*512]
 *   double u0x,u0y,u0z,u1x,u1y,u1z     [nchunks*512] each (speed buffers 0 and 1)
 *   double ax,ay,az                    [nchunks*512] each (acceleration)
 *   double p                           [nchunks*512]
 *   uint8  flags[nchunks*512]          bit0..2 const face x,y,z; bit3 no-delete
 *   uint8  type[nchunks*512]           0 air, 1 fluid, 2 solid, 3 inflow, 4 interior
 *   int32  layer[nchunks*512]          -1 = empty
 *   int32  id[nchunks*512]             solver numbering (-1 = none)
 *   int32  depth[nchunks*512]          distance to the surface (-1 = empty),
 *                                      src/Data_Grid_Depth_Empty.h:6-14
 *   double pos[nparticles][3]
 * Cell offset inside a chunk is x + 8y + 64z (src/Offset.h:14-24).
 */
#ifndef MAC_ORACLE_STATE_FORMAT_H
#define MAC_ORACLE_STATE_FORMAT_H

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MAC_BRICK 8
#define MAC_BRICK_CELLS 512
#define MAC_AIR 0
#define MAC_FLUID 1
#define MAC_SOLID 2
#define MAC_INFLOW 3
#define MAC_INTERIOR 4
#define MAC_FLAG_NODELETE 8

typedef struct {
  char magic[8];           /* "MACST002" */
  int64_t nchunks;
  int64_t nparticles;
  double h[3];
  double t, dt, cfl_factor, dt_min, dt_max, gravity;
  int32_t gravity_axis;    /* 1..3 */
  int32_t layer_max;
  uint64_t step;           /* refill seed counter */
  int32_t interp_symmetric;
  int32_t reserved_i;
  double viscosity;        /* Data_Viscosity::m_viscosity (0: inviscid) */
  int32_t depth_mode;      /* 1: the depth composition of the topology (Interior cells) */
  int32_t depth_max, depth_interior, depth_remove; /* Policy_Depth(max, interior, remove) */
  int32_t refill_cube;     /* 0: Jitter8 refill; n >= 1: Policy_Add_Particle_Cube(n) */
  int32_t reserved_j;
  uint8_t reserved[256 - 8 - 16 - 24 - 48 - 8 - 8 - 8 - 8 - 24];
} mac_state_header;

typedef struct {
  mac_state_header hdr;
  int32_t* keys;
  uint8_t* exists;
  double* u[2][3];
  double* acc[3];
  double* p;
  uint8_t* flags;
  uint8_t* type;
  int32_t* layer;
  int32_t* id;
  int32_t* depth;
  double* pos;
} mac_state_file;

static inline void mac_state_alloc(mac_state_file* s, int64_t nchunks, int64_t np) {
  size_t nc = (size_t)nchunks * MAC_BRICK_CELLS;
  s->keys = (int32_t*)calloc((size_t)nchunks * 3 + 1, 4);
  s->exists = (uint8_t*)calloc(nc + 1, 1);
  for (int b = 0; b < 2; ++b)
    for (int i = 0; i < 3; ++i) s->u[b][i] = (double*)calloc(nc + 1, 8);
  for (int i = 0; i < 3; ++i) s->acc[i] = (double*)calloc(nc + 1, 8);
  s->p = (double*)calloc(nc + 1, 8);
  s->flags = (uint8_t*)calloc(nc + 1, 1);
  s->type = (uint8_t*)calloc(nc + 1, 1);
  s->layer = (int32_t*)calloc(nc + 1, 4);
  s->id = (int32_t*)calloc(nc + 1, 4);
  s->depth = (int32_t*)calloc(nc + 1, 4);
  s->pos = (double*)calloc((size_t)np * 3 + 1, 8);
}

static inline void mac_state_free(mac_state_file* s) {
  free(s->keys); free(s->exists);
  for (int b = 0; b < 2; ++b)
    for (int i = 0; i < 3; ++i) free(s->u[b][i]);
  for (int i = 0; i < 3; ++i) free(s->acc[i]);
  free(s->p); free(s->flags); free(s->type); free(s->layer); free(s->id); free(s->depth); free(s->pos);
  memset(s, 0, sizeof(*s));
}

static inline int mac_state_io_(FILE* f, void* p, size_t sz, size_t n, int wr) {
  if (n == 0) return 0;
  size_t r = wr ? fwrite(p, sz, n, f) : fread(p, sz, n, f);
  return r == n ? 0 : -1;
}

static inline int mac_state_rw_(FILE* f, mac_state_file* s, int wr) {
  size_t nc = (size_t)s->hdr.nchunks * MAC_BRICK_CELLS;
  int e = 0;
  e |= mac_state_io_(f, s->keys, 4, (size_t)s->hdr.nchunks * 3, wr);
  e |= mac_state_io_(f, s->exists, 1, nc, wr);
  for (int b = 0; b < 2; ++b)
    for (int i = 0; i < 3; ++i) e |= mac_state_io_(f, s->u[b][i], 8, nc, wr);
  for (int i = 0; i < 3; ++i) e |= mac_state_io_(f, s->acc[i], 8, nc, wr);
  e |= mac_state_io_(f, s->p, 8, nc, wr);
  e |= mac_state_io_(f, s->flags, 1, nc, wr);
  e |= mac_state_io_(f, s->type, 1, nc, wr);
  e |= mac_state_io_(f, s->layer, 4, nc, wr);
  e |= mac_state_io_(f, s->id, 4, nc, wr);
  e |= mac_state_io_(f, s->depth, 4, nc, wr);
  e |= mac_state_io_(f, s->pos, 8, (size_t)s->hdr.nparticles * 3, wr);
  return e;
}

static inline int mac_state_read(const char* path, mac_state_file* s) {
  FILE* f = fopen(path, "rb");
  if (!f) return -1;
  mac_state_header h;
  if (fread(&h, sizeof(h), 1, f) != 1 || memcmp(h.magic, "MACST002", 8) != 0) { fclose(f); return -1; }
  mac_state_alloc(s, h.nchunks, h.nparticles);
  s->hdr = h;
  int e = mac_state_rw_(f, s, 0);
  fclose(f);
  return e;
}

static inline int mac_state_write(const char* path, mac_state_file* s) {
  FILE* f = fopen(path, "wb");
  if (!f) return -1;
  memcpy(s->hdr.magic, "MACST002", 8);
  int e = fwrite(&s->hdr, sizeof(s->hdr), 1, f) == 1 ? 0 : -1;
  e |= mac_state_rw_(f, s, 1);
  fclose(f);
  return e;
}

/* Counter-based jitter for the 8-particles-per-cell refill policy. Particle s of
 * cell k sits at ((k_i + o_i) + j_i) * h_i with o_i = -1/4 or +1/4 (bit i of s)
 * and j_i uniform in (-0.2495, 0.2495), drawn from splitmix64 of (seed, k, s, i).
 * The device implementation in mac_b200/csrc computes the same bits. */
static inline uint64_t mac_oracle_mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static inline void mac_jitter8_position(uint64_t seed, int kx, int ky, int kz, int s,
                                        double hx, double hy, double hz, double out[3]) {
  int k[3] = {kx, ky, kz};
  double hh[3] = {hx, hy, hz};
  uint64_t base = mac_oracle_mix64(seed ^ mac_oracle_mix64(((uint64_t)(uint32_t)kx) |
                                                           ((uint64_t)(uint32_t)ky << 32)));
  base = mac_oracle_mix64(base ^ (uint64_t)(uint32_t)kz);
  for (int i = 0; i < 3; ++i) {
    uint64_t r = mac_oracle_mix64(base ^ (uint64_t)(s * 3 + i + 1));
    double u = (double)(r >> 11) * (1.0 / 9007199254740992.0);
    double j = (u - 0.5) * 0.499;
    double o = ((s >> i) & 1) ? 0.25 : -0.25;
    out[i] = (((double)k[i] + o) + j) * hh[i];
  }
}

#endif
