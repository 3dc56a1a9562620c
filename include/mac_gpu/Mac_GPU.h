/* C++ drop-in layer over the C-ABI (include/mac_gpu.h) for a Mac world.
 *
 * The reference composes a world from header templates and runs it through
 * algorithm classes of one shape (src/Algorithms_*.h):
 *     template<class DataRef, class Policy> class Algorithms_X : public Policy
 *     { Algorithms_X(DataRef data, const Policy& pol); void Do(); };
 * grouped with Algorithms<...> and Policies<...> (src/Algorithms.h, src/Policies.h).
 * The classes below keep that shape, with a _GPU suffix, so a reference main()
 * swaps them in for the host algorithms they name:
 *
 *   Policy_Solve_Linear_GPU          for Policy_Solve_Linear_Umfpack
 *                                    (src/Policy_Solve_Linear_Umfpack.h:23-70), used by
 *                                    the unmodified Algorithms_Solve_Pressure;
 *   Algorithms_<X>_GPU<DataRef, Policy_Mac_GPU<DataRef>>
 *                                    for Algorithms_<X> of the pipeline-A step
 *                                    (test/TestJetDEau_Basic.cpp:325-441).
 *
 * The world lives on the device between GPU algorithms. Mac_GPU_Session packs
 * the reference's chunk grid into a mac_host_state on the first GPU algorithm
 * and unpacks it again when Algorithms_To_Host_GPU runs (before any host
 * algorithm, output or checkpoint that reads the world). Requires a chunk edge
 * N = 8 (the device bricks are 8^3) and the four-material cell type
 * (src/Data_CellType_Fluid_Air_Solid_Inflow.h), or the cell type of the depth
 * composition (src/Data_CellType_Fluid_Air_Solid_Inflow_Interior_0_Pres.h, whose
 * 0-pressure material no algorithm sets) with a Data_Chunk_Depth: the session
 * detects the interior material and the depth chunk and carries both, so
 * mac_params.depth_mode / .pipeline worlds (test/Jet3.cpp) run through the
 * same classes plus Algorithms_RungeKutta_all_GPU.
 *
 * Errors follow the reference's convention for its solver policy
 * (src/Policy_Solve_Linear_Umfpack.h:15-21): the status is printed and the run
 * goes on; Mac_GPU_Session::Status() keeps the first failure for the caller.
 * C++11, header only; link with libmac_gpu.so.
 */
#ifndef MAC_GPU_HPP
#define MAC_GPU_HPP

#include <cstdint>
#include <iostream>
#include <map>
#include <memory>
#include <tuple>
#include <type_traits>
#include <vector>

#include "../mac_gpu.h"

namespace mac_gpu_detail {

inline int report(int rc, const char* what) {
  if (rc != MAC_OK) std::cout << "mac_gpu: " << what << " failed: " << mac_error_string(rc) << std::endl;
  return rc;
}

inline int chunk_of(int v) { return v >= 0 ? v / MAC_BRICK_EDGE : (v + 1) / MAC_BRICK_EDGE - 1; }

/* Whether the cell type's material enum has the interior material
 * (src/Data_CellType_Fluid_Air_Solid_Inflow_Interior_0_Pres.h). */
template <class M, class = void>
struct has_interior : std::false_type {};
template <class M>
struct has_interior<M, decltype((void)M::Interior)> : std::true_type {};

template <class M>
uint8_t interior_or_air(M m, std::true_type) { return m == M::Interior ? (uint8_t)MAC_CELL_INTERIOR : (uint8_t)MAC_CELL_AIR; }
template <class M>
uint8_t interior_or_air(M, std::false_type) { return MAC_CELL_AIR; }
template <class M>
M interior_material(std::true_type) { return M::Interior; }
template <class M>
M interior_material(std::false_type) { return M::Air; }

/* Material to MAC_CELL_* (MaterialToInt, src/Data_CellType_Fluid_Air_Solid_Inflow.tpp:3-18). */
template <class M>
uint8_t to_code(M m) {
  if (m == M::Fluid) return MAC_CELL_FLUID;
  if (m == M::Solid) return MAC_CELL_SOLID;
  if (m == M::Inflow) return MAC_CELL_INFLOW;
  return interior_or_air(m, has_interior<M>());
}
template <class M>
M from_code(uint8_t c) {
  switch (c) {
    case MAC_CELL_FLUID: return M::Fluid;
    case MAC_CELL_SOLID: return M::Solid;
    case MAC_CELL_INFLOW: return M::Inflow;
    case MAC_CELL_INTERIOR: return interior_material<M>(has_interior<M>());
    default: return M::Air;
  }
}

/* Whether the world's chunk carries a depth (src/Data_Chunk_Depth.h). */
template <class C, class = void>
struct has_depth : std::false_type {};
template <class C>
struct has_depth<C, decltype((void)std::declval<C&>().Depth_GetPointer())> : std::true_type {};

template <class C>
void pack_depth(C& ch, int32_t* d, std::true_type) {
  for (int o = 0; o < MAC_BRICK_CELLS; ++o) d[o] = ch.Depth_GetPointer()[o].GetDepth();
}
template <class C>
void pack_depth(C&, int32_t*, std::false_type) {}
template <class C>
void unpack_depth(C& ch, const int32_t* d, std::true_type) {
  for (int o = 0; o < MAC_BRICK_CELLS; ++o) ch.Depth_GetPointer()[o].SetDepth(d[o]);
}
template <class C>
void unpack_depth(C&, const int32_t*, std::false_type) {}

}  // namespace mac_gpu_detail

/* Drop-in for Policy_Solve_Linear_Umfpack: same three member functions, same
 * argument meaning (CSC arrays owned by the caller; the policy owns only its
 * device copy). FP64 Jacobi-PCG on the device to relative residual rtol. */
class Policy_Solve_Linear_GPU {
  std::shared_ptr<void> m_ctx;
  int m_n = 0;

 public:
  explicit Policy_Solve_Linear_GPU(double rtol = 1e-14, int max_iters = 100000, int device = 0) {
    mac_params p;
    mac_default_params(&p);
    p.rtol = rtol;
    p.max_iters = max_iters;
    p.device = device;
    p.max_bricks = 1;
    p.max_particles = 1;
    void* c = nullptr;
    if (mac_gpu_detail::report(mac_ctx_create(&p, &c), "mac_ctx_create") == MAC_OK)
      m_ctx = std::shared_ptr<void>(c, [](void* q) { mac_ctx_destroy(q); });
  }
  void Solve_Linear_FactorizeMatrice(int n, int* offset, int* indice, double* value) {
    if (!m_ctx) return;
    m_n = n;
    mac_gpu_detail::report(mac_csc_factorize(m_ctx.get(), n, offset, indice, value), "mac_csc_factorize");
  }
  void Solve_Linear(int n, int* offset, int* indice, double* value, double* b, double* res) {
    (void)offset;
    (void)indice;
    (void)value;
    if (!m_ctx || n != m_n) {
      std::cout << "mac_gpu: Solve_Linear without a matching Solve_Linear_FactorizeMatrice" << std::endl;
      return;
    }
    mac_gpu_detail::report(mac_csc_solve(m_ctx.get(), n, b, res), "mac_csc_solve");
  }
  void Solve_Linear_Clean() {
    if (m_ctx) mac_gpu_detail::report(mac_csc_clean(m_ctx.get()), "mac_csc_clean");
    m_n = 0;
  }
  /* Iterations of the last solve (no counterpart in the Umfpack policy). */
  int Iterations() const {
    mac_stats s;
    if (!m_ctx || mac_get_stats(m_ctx.get(), &s) != MAC_OK) return -1;
    return s.iterations;
  }
};

/* Owns the device context and moves the world between the reference's chunk
 * grid and the device. DataRef is the reference's DataRef<...> of the world. */
template <class DataRef>
class Mac_GPU_Session {
  typedef typename DataRef::type_data_struct::type_Data_Grid type_Data_Grid;
  typedef typename type_Data_Grid::type_key type_key;
  typedef typename DataRef::type_data_struct::type_Data_Topology type_Data_Topology;
  typedef typename type_Data_Topology::type_particle_list type_particle_list;
  typedef typename type_Data_Topology::type_particle type_particle;
  typedef typename type_particle::type_data_vector type_data_vector;
  typedef typename std::remove_reference<decltype(
      std::declval<type_Data_Grid&>().DirectAcessChunk(std::declval<const type_key&>()))>::type type_chunk;
  typedef mac_gpu_detail::has_depth<type_chunk> type_has_depth;
  typedef typename type_Data_Grid::type_data::type_chunk_speed type_chunk_speed;

  DataRef m_data;
  std::vector<std::tuple<int, int, int>> m_order;  // chunk keys (x, y, z) in the device's brick order
  void* m_ctx = nullptr;
  bool m_on_device = false;
  int m_status = MAC_OK;
  uint64_t m_step;

  int keep(int rc, const char* what) {
    mac_gpu_detail::report(rc, what);
    if (rc != MAC_OK && m_status == MAC_OK) m_status = rc;
    return rc;
  }

  struct Host {
    std::vector<int32_t> keys, layer, depth;
    std::vector<uint8_t> exists, flags, type;
    std::vector<double> f[10], pos;  // u0x..u1z, ax..az, p
    mac_host_state view{};
    void size(int64_t nb, int64_t np) {
      size_t nc = (size_t)nb * MAC_BRICK_CELLS;
      keys.assign(3 * (size_t)nb, 0);
      layer.assign(nc, -1);
      exists.assign(nc, 0);
      flags.assign(nc, 0);
      type.assign(nc, 0);
      for (int i = 0; i < 10; ++i) f[i].assign(nc, 0.0);
      pos.assign(3 * (size_t)np, 0.0);
      view.nbricks = nb;
      view.nparticles = np;
      view.keys = keys.data();
      view.exists = exists.data();
      for (int b = 0; b < 2; ++b)
        for (int i = 0; i < 3; ++i) view.u[b][i] = f[3 * b + i].data();
      for (int i = 0; i < 3; ++i) view.acc[i] = f[6 + i].data();
      view.p = f[9].data();
      view.flags = flags.data();
      view.type = type.data();
      view.layer = layer.data();
      view.pos = pos.data();
      depth.assign(type_has_depth::value ? nc : 0, -1);
      view.depth = type_has_depth::value ? depth.data() : nullptr;
    }
  };

 public:
  /* step: the refill counter that seeds the inflow particle jitter. */
  Mac_GPU_Session(DataRef data, const mac_params& prm, uint64_t step = 0) : m_data(data), m_step(step) {
    keep(mac_ctx_create(&prm, &m_ctx), "mac_ctx_create");
  }
  ~Mac_GPU_Session() {
    if (m_ctx) mac_ctx_destroy(m_ctx);
  }
  Mac_GPU_Session(const Mac_GPU_Session&) = delete;
  Mac_GPU_Session& operator=(const Mac_GPU_Session&) = delete;

  void* Context() const { return m_ctx; }
  int Status() const { return m_status; }
  uint64_t Step() const { return m_step; }
  bool OnDevice() const { return m_on_device; }

  /* Packs the host world and uploads it (no-op when the device copy is current). */
  int ToDevice() {
    if (!m_ctx) return MAC_ERR_INVALID;
    if (m_on_device) return MAC_OK;
    int rc = Upload();
    m_on_device = rc == MAC_OK;
    return rc;
  }

  /* Packs the host world and uploads it; the host copy stays the master. */
  int Upload() {
    if (!m_ctx) return MAC_ERR_INVALID;
    type_Data_Grid& grid = m_data.m_data.GetGridData();
    std::map<std::tuple<int, int, int>, int64_t> chunks;
    for (auto it = grid.begin(); it != grid.end(); ++it) {
      type_key k = it.key();
      auto ck = std::make_tuple(mac_gpu_detail::chunk_of(k.Get(3)), mac_gpu_detail::chunk_of(k.Get(2)),
                                mac_gpu_detail::chunk_of(k.Get(1)));
      if (!chunks.count(ck)) chunks.emplace(ck, 0);
    }
    type_particle_list& plist = m_data.m_data.GetTopologyData().GetRefToParticleList();
    Host h;
    h.size((int64_t)chunks.size(), (int64_t)plist.size());
    int64_t b = 0;
    m_order.clear();
    for (auto& kv : chunks) {
      int cx = std::get<2>(kv.first), cy = std::get<1>(kv.first), cz = std::get<0>(kv.first);
      m_order.emplace_back(cx, cy, cz);
      h.keys[3 * b] = cx;
      h.keys[3 * b + 1] = cy;
      h.keys[3 * b + 2] = cz;
      type_key ckey;
      ckey.Set(1, cx);
      ckey.Set(2, cy);
      ckey.Set(3, cz);
      auto& ch = grid.DirectAcessChunk(ckey);
      for (int o = 0; o < MAC_BRICK_CELLS; ++o) {
        size_t i = (size_t)b * MAC_BRICK_CELLS + o;
        h.exists[i] = ch.GetChunk_Bool_Array()[o] ? 1 : 0;
        for (int s = 0; s < 2; ++s)
          for (int d = 1; d <= 3; ++d) h.f[3 * s + d - 1][i] = ch.Speed_GetPointer(s)[o].Get(d);
        for (int d = 1; d <= 3; ++d) h.f[6 + d - 1][i] = ch.Acceleration_GetPointer(0)[o].Get(d);
        h.f[9][i] = ch.Pressure_GetPointer()[o].Pressure_Get().Get();
        uint8_t fl = 0;
        for (int d = 1; d <= 3; ++d)
          if (ch.Speed_GetPointer(0)[o].Get_Const(d)) fl |= (uint8_t)(1u << (d - 1));
        auto& ct = ch.CellType_GetPointer()[o];
        if (ct.GetIsNoDelete()) fl |= MAC_FLAG_NODELETE;
        h.flags[i] = fl;
        h.type[i] = mac_gpu_detail::to_code(ct.m_mat);
        h.layer[i] = ch.Layer_GetPointer()[o].GetLayer();
      }
      if (type_has_depth::value)
        mac_gpu_detail::pack_depth(ch, h.depth.data() + (size_t)b * MAC_BRICK_CELLS, type_has_depth());
      ++b;
    }
    int64_t q = 0;
    for (auto it = plist.begin(); it != plist.end(); ++it, ++q) {
      const type_data_vector& v = (*it).GetParticlePos();
      for (int d = 1; d <= 3; ++d) h.pos[3 * q + d - 1] = v.Get(d);
    }
    auto& timing = m_data.m_data.GetTimingData();
    h.view.t = timing.m_t;
    h.view.dt = timing.m_dt;
    h.view.step = m_step;
    return keep(mac_upload_state(m_ctx, &h.view), "mac_upload_state");
  }

  /* The projection with the world on the host, for the reference's own
   * integrators (Algorithms_Solve_Pressure_GPU). Init uploads the world and
   * builds the device system; each projection uploads the field it projects
   * (the speed buffer type_chunk_speed::ispeed, or the acceleration when
   * SetAccel_Instead_Speed(true) is in force, src/Data_Chunk_Speed.h:150-171),
   * runs Divergence_Projection on the device and writes the projected field
   * and the pressure back into the chunk grid. */
  int ProjectionInit() {
    if (m_on_device && ToHost()) return m_status;
    int rc = Upload();
    return rc ? rc : keep(mac_pressure_init(m_ctx), "mac_pressure_init");
  }
  int ProjectionRun() {
    if (!m_ctx) return MAC_ERR_INVALID;
    const int ispeed = type_chunk_speed::ispeed;
    const bool accel = type_chunk_speed::GetAccel_Instead_Speed();
    const size_t nc = m_order.size() * (size_t)MAC_BRICK_CELLS;
    std::vector<double> buf(nc);
    const int sfield = MAC_FIELD_U0X + 3 * ispeed;
    const int target = accel ? (int)MAC_FIELD_AX : sfield;
    int rc = MAC_OK;
    for (int d = 1; d <= 3 && !rc; ++d) {
      Field(ispeed, d, buf.data(), true);
      rc = keep(mac_upload_field(m_ctx, sfield + d - 1, buf.data()), "mac_upload_field");
      if (!rc && accel) {
        Field(-1, d, buf.data(), true);
        rc = keep(mac_upload_field(m_ctx, MAC_FIELD_AX + d - 1, buf.data()), "mac_upload_field");
      }
    }
    if (rc) return rc;
    const int st = keep(mac_pressure_divergence_projection(m_ctx, ispeed, accel ? 1 : 0),
                        "mac_pressure_divergence_projection");
    if (st && st != MAC_ERR_NOT_CONVERGED) return st;
    for (int d = 1; d <= 3 && !rc; ++d) {
      rc = keep(mac_download_field(m_ctx, target + d - 1, buf.data()), "mac_download_field");
      if (!rc) Field(accel ? -1 : ispeed, d, buf.data(), false);
    }
    if (!rc) rc = keep(mac_download_field(m_ctx, MAC_FIELD_P, buf.data()), "mac_download_field");
    if (!rc) Pressure(buf.data());
    return rc ? rc : st;
  }
  int ProjectionEnd() { return keep(mac_pressure_end(m_ctx), "mac_pressure_end"); }

 private:
  /* Component d of speed buffer s (s = -1: the acceleration) of every cell, in
   * the device's brick order: packed into v (to_device) or written from it. */
  void Field(int s, int d, double* v, bool to_device) {
    type_Data_Grid& grid = m_data.m_data.GetGridData();
    for (size_t b = 0; b < m_order.size(); ++b) {
      type_key ckey;
      ckey.Set(1, std::get<0>(m_order[b]));
      ckey.Set(2, std::get<1>(m_order[b]));
      ckey.Set(3, std::get<2>(m_order[b]));
      auto& ch = grid.DirectAcessChunk(ckey);
      auto* f = s < 0 ? ch.Acceleration_GetPointer(0) : ch.Speed_GetPointer(s);
      for (int o = 0; o < MAC_BRICK_CELLS; ++o) {
        double& x = v[b * MAC_BRICK_CELLS + o];
        if (to_device) x = f[o].Get(d);
        else f[o].m_speed.Set(d, x);
      }
    }
  }
  void Pressure(const double* v) {
    type_Data_Grid& grid = m_data.m_data.GetGridData();
    for (size_t b = 0; b < m_order.size(); ++b) {
      type_key ckey;
      ckey.Set(1, std::get<0>(m_order[b]));
      ckey.Set(2, std::get<1>(m_order[b]));
      ckey.Set(3, std::get<2>(m_order[b]));
      auto& ch = grid.DirectAcessChunk(ckey);
      for (int o = 0; o < MAC_BRICK_CELLS; ++o) ch.Pressure_GetPointer()[o].Pressure_Set(v[b * MAC_BRICK_CELLS + o]);
    }
  }

 public:

  /* Downloads the device world into the reference's chunk grid: chunks and
   * cells erased on the device are erased on the host, live chunks get all
   * 512 slots (erased cells of a live chunk keep their data, as in the
   * reference), and the particle list is replaced. */
  int ToHost() {
    if (!m_ctx) return MAC_ERR_INVALID;
    if (!m_on_device) return MAC_OK;
    int64_t nb = 0, np = 0;
    int rc = keep(mac_query_sizes(m_ctx, &nb, &np), "mac_query_sizes");
    if (rc) return rc;
    Host h;
    h.size(nb, np);
    if ((rc = keep(mac_download_state(m_ctx, &h.view), "mac_download_state"))) return rc;
    type_Data_Grid& grid = m_data.m_data.GetGridData();
    std::map<std::tuple<int, int, int>, int64_t> live;
    for (int64_t b = 0; b < nb; ++b) live.emplace(std::make_tuple(h.keys[3 * b], h.keys[3 * b + 1], h.keys[3 * b + 2]), b);
    auto it = grid.begin();
    while (it != grid.end()) {
      type_key k = it.key();
      int x = k.Get(1), y = k.Get(2), z = k.Get(3);
      auto f = live.find(std::make_tuple(mac_gpu_detail::chunk_of(x), mac_gpu_detail::chunk_of(y),
                                         mac_gpu_detail::chunk_of(z)));
      int o = (x - MAC_BRICK_EDGE * mac_gpu_detail::chunk_of(x)) +
              MAC_BRICK_EDGE * ((y - MAC_BRICK_EDGE * mac_gpu_detail::chunk_of(y)) +
                                MAC_BRICK_EDGE * (z - MAC_BRICK_EDGE * mac_gpu_detail::chunk_of(z)));
      if (f == live.end() || !h.exists[(size_t)f->second * MAC_BRICK_CELLS + o])
        it = grid.erase(it);
      else
        ++it;
    }
    for (auto& kv : live) {
      int64_t b = kv.second;
      type_key k0, ckey;
      for (int d = 1; d <= 3; ++d) {
        k0.Set(d, h.keys[3 * b + d - 1] * MAC_BRICK_EDGE);
        ckey.Set(d, h.keys[3 * b + d - 1]);
      }
      grid[k0];  // creates the chunk when it is new
      auto& ch = grid.DirectAcessChunk(ckey);
      for (int o = 0; o < MAC_BRICK_CELLS; ++o) {
        size_t i = (size_t)b * MAC_BRICK_CELLS + o;
        ch.GetChunk_Bool_Array()[o] = h.exists[i] != 0;
        for (int s = 0; s < 2; ++s)
          for (int d = 1; d <= 3; ++d) ch.Speed_GetPointer(s)[o].m_speed.Set(d, h.f[3 * s + d - 1][i]);
        for (int d = 1; d <= 3; ++d) ch.Acceleration_GetPointer(0)[o].m_speed.Set(d, h.f[6 + d - 1][i]);
        auto& s0 = ch.Speed_GetPointer(0)[o];
        for (int d = 1; d <= 3; ++d) {
          if (h.flags[i] & (1u << (d - 1)))
            s0.Set_Const(d);
          else
            s0.Set_None_Const(d);
        }
        ch.Pressure_GetPointer()[o].Pressure_Set(h.f[9][i]);
        auto& ct = ch.CellType_GetPointer()[o];
        typedef typename std::remove_reference<decltype(ct)>::type::Material_Type Mat;
        ct.m_mat = mac_gpu_detail::from_code<Mat>(h.type[i]);
        ct.SetIsNoDelete((h.flags[i] & MAC_FLAG_NODELETE) != 0);
        ch.Layer_GetPointer()[o].SetLayer(h.layer[i]);
      }
      if (type_has_depth::value)
        mac_gpu_detail::unpack_depth(ch, h.depth.data() + (size_t)b * MAC_BRICK_CELLS, type_has_depth());
    }
    type_particle_list& plist = m_data.m_data.GetTopologyData().GetRefToParticleList();
    while (plist.size()) plist.pop_back();
    for (int64_t q = 0; q < np; ++q) {
      type_data_vector v;
      for (int d = 1; d <= 3; ++d) v.Set(d, h.pos[3 * q + d - 1]);
      plist.push_back(type_particle(v));
    }
    auto& timing = m_data.m_data.GetTimingData();
    timing.m_t = h.view.t;
    timing.m_dt = h.view.dt;
    m_step = h.view.step;
    m_on_device = false;
    return MAC_OK;
  }

  /* Runs one C-ABI stage on the device copy of the world. */
  template <class F>
  int Run(F stage, const char* what) {
    int rc = ToDevice();
    if (rc) return rc;
    return keep(stage(m_ctx), what);
  }
};

/* The policy the GPU algorithms take: a shared handle on the session, so the
 * copies the algorithm classes make (they derive from their policy) all reach
 * the same device world. */
template <class DataRef>
class Policy_Mac_GPU {
 public:
  std::shared_ptr<Mac_GPU_Session<DataRef>> m_session;
  Policy_Mac_GPU(DataRef data, const mac_params& prm, uint64_t step = 0)
      : m_session(std::make_shared<Mac_GPU_Session<DataRef>>(data, prm, step)) {}
  Mac_GPU_Session<DataRef>& Session() const { return *m_session; }
};

#define MAC_GPU_ALGORITHM(NAME, CALL)                                               \
  template <class DataRef, class Policy>                                           \
  class NAME : public Policy {                                                     \
   public:                                                                         \
    NAME(DataRef data, const Policy& pol) : Policy(pol) { (void)data; }            \
    void Do() {                                                                    \
      this->Session().Run([](void* c) { return CALL; }, #NAME);                    \
    }                                                                              \
  };

/* src/Algorithms_Initialize_MacCell.h:15-21 */
MAC_GPU_ALGORITHM(Algorithms_Initialize_MacCell_GPU, mac_initialize_maccell(c))
/* src/Algorithms_Layer_Initial_With_Particle.h:20-34 */
MAC_GPU_ALGORITHM(Algorithms_Layer_Initial_With_Particle_GPU, mac_layer_initial_with_particle(c))
/* src/Algorithms_Create_Fluid_Particle.h:19-33 */
MAC_GPU_ALGORITHM(Algorithms_Create_Fluid_Particle_GPU, mac_create_fluid_particle(c))
/* src/Algorithms_Update_CellType_Layer.h:22-89 */
MAC_GPU_ALGORITHM(Algorithms_Update_CellType_Layer_GPU, mac_update_celltype_layer(c))
/* src/Algorithms_Delete_MacCell.h:22-44 */
MAC_GPU_ALGORITHM(Algorithms_Delete_MacCell_GPU, mac_delete_maccell(c))
/* src/Algorithms_Calculate_Time_Step.h:35-66 */
MAC_GPU_ALGORITHM(Algorithms_Calculate_Time_Step_GPU, mac_calculate_time_step(c, nullptr))
/* The whole Algorithms<Initialize..., Calculate_Time_Step> group of
 * test/TestJetDEau_Basic.cpp:325-326, refill counter advanced first. */
MAC_GPU_ALGORITHM(Algorithms_Topology_GPU, mac_topology_rebuild(c))
/* acc = 0, then Algorithms<Algorithms_Gravity, Algorithms_Convection> on speed 0
 * (src/Algorithms_Gravity.h:15-28, src/Algorithms_Convection.h:18-37) */
MAC_GPU_ALGORITHM(Algorithms_Gravity_Convection_GPU, mac_forces(c, 0))
/* src/Algorithms_Do_Pressure.h:16-21 on speed 0 */
MAC_GPU_ALGORITHM(Algorithms_Do_Pressure_GPU, mac_pressure_project(c, 0))
/* src/Algorithms_RungeKutta_RK2_TVD.h:20-66 */
MAC_GPU_ALGORITHM(Algorithms_RungeKutta_RK2_TVD_GPU, mac_rk2tvd(c))
/* src/Algorithms_Extrapolate.h:25-233 */
MAC_GPU_ALGORITHM(Algorithms_Extrapolate_GPU, mac_extrapolate(c))
/* src/Algorithm_Extrapolate_Boundary_Condition.h:454-975 on speed 0, in the device's
 * fixed colour order (mac_extrapolate_boundary_condition) */
MAC_GPU_ALGORITHM(Algorithm_Extrapolate_Boundary_Condition_GPU, mac_extrapolate_boundary_condition(c, 0))
/* src/Algorithms_Move_Particles.h:22-36 */
MAC_GPU_ALGORITHM(Algorithms_Move_Particles_GPU, mac_move_particles(c))
/* src/Algorithms_RungeKutta_all.h:35-156 with the policy of test/Jet3.cpp:642-675
 * (a context created with mac_params.pipeline = 1) */
MAC_GPU_ALGORITHM(Algorithms_RungeKutta_all_GPU, mac_rungekutta_all(c))
/* One step: pipeline A, test/TestJetDEau_Basic.cpp:434-441 (t += dt included),
 * or, with mac_params.pipeline = 1, pipeline B, test/Jet3.cpp:720-726. */
MAC_GPU_ALGORITHM(Algorithms_Step_GPU, mac_step(c))

#undef MAC_GPU_ALGORITHM

/* Algorithms_Solve_Pressure at its composable interface
 * (src/Algorithms_Solve_Pressure.h:44,158,168): Init_Iteration,
 * Divergence_Projection and End_Iteration on the device, for the reference's
 * own integrators, which call them through Policy:: between host loops over
 * the speed buffers (src/Algorithms_RungeKutta_RK2_TVD.h:29,50,60-61), and for
 * Algorithms_Do_Pressure (src/Algorithms_Do_Pressure.h:16-21). The world
 * stays on the host; each projection moves only the field it projects and
 * the pressure. In place of the reference's
 *     Policies<type_alg_solve_grid, Algorithms_Solve_Pressure<DataRef, type_pol_pres>>
 * a world composes
 *     Policies<type_alg_solve_grid, Algorithms_Solve_Pressure_GPU<DataRef, Policy_Mac_GPU<DataRef>>>. */
template <class DataRef, class Policy>
class Algorithms_Solve_Pressure_GPU : public Policy {
 public:
  Algorithms_Solve_Pressure_GPU(DataRef data, const Policy& pol) : Policy(pol) { (void)data; }
  void Init_Iteration() { this->Session().ProjectionInit(); }
  void Divergence_Projection() { this->Session().ProjectionRun(); }
  void End_Iteration() { this->Session().ProjectionEnd(); }
};

/* Brings the device world back into the reference's chunk grid; put it before
 * any host algorithm (output, checkpoint) that reads the world. */
template <class DataRef, class Policy>
class Algorithms_To_Host_GPU : public Policy {
 public:
  Algorithms_To_Host_GPU(DataRef data, const Policy& pol) : Policy(pol) { (void)data; }
  void Do() { this->Session().ToHost(); }
};

#endif
