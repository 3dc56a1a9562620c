// Reference world runner: composes the UNMODIFIED Mac headers (pipeline-A step of
// test/TestJetDEau_Basic.cpp:145-446) into one concrete world, loads a state file,
// runs a named stage or whole steps, and writes the resulting state.
//
// Test infrastructure only: it is compiled from the reference sources into
// oracle/_ref/ by oracle/Makefile and is used to pin the C restatement
// (oracle/mac_oracle.c) and as the timed CPU baseline. Nothing in the product
// links or runs it.
//
// Deviations from test/TestJetDEau_Basic.cpp, all forced by the environment:
//  * chunk edge N = 8 (the device bricks are 8^3; test/Jet3.cpp:299 also uses 8),
//  * Policy_Solve_Linear_Umfpack (src/Policy_Solve_Linear_Umfpack.h:23-70) is
//    replaced by Policy_Solve_Linear_OracleCG below with the same three member
//    functions, because libumfpack is not installed: FP64 Jacobi-CG to a relative
//    residual of 1e-14 (a direct-solve stand-in; tests pin it against a sparse
//    LU on the same CSC arrays),
//  * Wind is not composed; viscosity (Algorithms_Viscosity and the Dirichlet
//    pressure of Algorithms_Solve_Pressure_Dirichlet, as test/Lateral_jet_3.cpp
//    composes them under VISCOSITY) only in the v* commands, with the
//    viscosity of the state header,
//  * prototype speed/pressure/layer/id are initialised explicitly (the reference
//    leaves them uninitialised: src/Physvector.tpp:8-10),
//  * inflow refill uses Policy_Add_Particle_Jitter8 (8 jittered particles per
//    cell, seeded by a counter-based hash shared with the oracle and the GPU)
//    or, when the state header asks for it, the reference's own
//    Policy_Add_Particle_Cube(n) (test/Jet3.cpp:509-510 uses n = 1).
//
// Built with -DMAC_DEPTH (oracle/_ref/mac_ref_depth) the world takes the cell
// type and topology of the depth composition of test/Jet3.cpp:326-386,503-549:
// Data_CellType_Fluid_Air_Solid_Inflow_Interior_0_Pres with
// Data_CellType_Domain_Fluid_Without_0_Pres, a depth per cell, Policy_Depth
// from the state header, and Initialize_Layer_And_Depth,
// Layer_Initial_With_Particle_Depth, Create_Fluid_Particle_Depth and
// Update_CellType_Layer_Depth in place of the four pipeline-A topology passes
// (the jet's own particle filter, Algorithm_DelParticle of test/Jet3.cpp:259-288,
// is not part of it).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <cmath>
#include <set>
#include <vector>
#include <string>
#include <chrono>
#include <fstream>
#include <iostream>
#include <unistd.h>

#include "Physvector.h"
#include "HashPhysvector.h"
#include "Neighbour_List_Empty.h"
#include "ChunkHashTable.h"
#include "Hook_Neighbour_List_Chunk.h"
#include "Data_Base_Dim_Type.h"
#include "Data_Staggered_Left.h"
#include "Data_Grid_Data.h"
#include "Data_Grid_Table.h"
#include "Data_Grid_Base_Spacing.h"
#include "Data_Viscosity.h"
#include "Data_CellType_Interface_Constant.h"
#include "Data_CellType_Fluid_Air_Solid_Inflow.h"
#include "Data_CellType_Domain_Fluid.h"
#include "Data_Grid_CellType_To_Grid_CellType.h"
#include "Data_Grid_Speed.h"
#include "Data_Grid_Pressure.h"
#include "Data_Grid_Layer.h"
#include "Data_Grid_Layer_Empty.h"
#include "Offset.h"
#include "Offset_Base.h"
#include "Offset_Base_Neighbour.h"
#include "Offset_Base_Pressure.h"
#include "Offset_Base_Speed.h"
#include "Offset_Base_CellType.h"
#include "Offset_Base_Layer.h"
#include "Offset_Base_Id_Cell.h"
#include "Data_Chunk.h"
#include "Data_Chunk_Pressure.h"
#include "Data_Chunk_CellType.h"
#include "Data_Chunk_Layer.h"
#include "Data_Chunk_Speed.h"
#include "Data_Chunk_Bool_Array.h"
#include "Data_Chunk_Id_Cell.h"
#include "Data_Topology.h"
#include "Data_Particle.h"
#include "Data_Particles_List.h"
#include "Data_Timing.h"
#include "Data_Timing_Time.h"
#include "Empty.h"
#include "Datas.h"
#include "DataRef.h"
#include "Policies.h"
#include "Algorithms.h"
#include "Policy_Layer_Max.h"
#include "Policy_Particle_To_Key.h"
#include "Policy_CheckDT.h"
#include "Policy_Gravity.h"
#include "Policy_Divergence.h"
#include "Policy_Gradiant.h"
#include "Policy_Von_Neumann_Boundary.h"
#include "Policy_Is_Inbound_Filling_Layer_CellType.h"
#include "Policy_Advance_ODE_RungeKutta.h"
#include "Policy_Speed_Interpolation_Linear_Symmetric.h"
#include "Policy_Speed_Interpolation_Linear.h"
#include "Policy_Upwind_1_Order.h"
#include "Policy_Convection_Apply_If.h"
#include "Policy_Pressure_If_Correction.h"
#include "Algorithms_Speed_Constant_Mirror.h"
#include "Algorithms_Solid_To_Const.h"
#include "Algorithms_Extrapolate.h"
#include "Algorithms_Initialize_MacCell.h"
#include "Algorithms_Create_Fluid_Particle.h"
#include "Algorithms_Layer_Initial_With_Particle.h"
#include "Algorithms_Calculate_Time_Step.h"
#include "Algorithms_Delete_MacCell.h"
#include "Algorithms_Update_CellType_Layer.h"
#include "Algorithms_Gravity.h"
#include "Algorithms_Solve_Pressure.h"
#include "Algorithms_Do_Pressure.h"
#include "Algorithms_Convection.h"
#include "Algorithms_Move_Particles.h"
#include "Algorithms_RungeKutta_RK2_TVD.h"
#include "Policy_Laplacian_Speed.h"
#include "Policy_Viscosity_Apply_If.h"
#include "Policy_Dirichlet_Boundary.h"
#include "Algorithms_Viscosity.h"
#include "Algorithms_Solve_Pressure_Dirichlet.h"
#include "Policy_Add_Particle_Cube.h"
#include "Policy_Is_In_Domain_Speed.h"
#include <cassert>  // src/Algorithm_Extrapolate_Boundary_Condition.h:193 uses assert without including it
#include "Algorithm_Extrapolate_Boundary_Condition.h"
#ifdef MAC_DEPTH
#include "Data_CellType_Fluid_Air_Solid_Inflow_Interior_0_Pres.h"
#include "Data_CellType_Domain_Fluid_Without_0_Pres.h"
#include "Data_Grid_Depth.h"
#include "Data_Grid_Depth_Empty.h"
#include "Data_Chunk_Depth.h"
#include "Offset_Base_Depth.h"
#include "Policy_Depth.h"
#include "Algorithms_Initialize_Layer_And_Depth.h"
#include "Algorithms_Layer_Initial_With_Particle_Depth.h"
#include "Algorithms_Create_Fluid_Particle_Depth.h"
#include "Algorithms_Update_CellType_Layer_Depth.h"
#endif
#ifdef MAC_PIPELINE_B
#include "Algorithms_Create_Interior_Depth.h"
#include "Algorithms_Solve_Pressure_Force.h"
#include "Algorithms_Accel_To_Speed.h"
#include "Policy_Move_Particle.h"
#include "Algorithms_RungeKutta_all.h"
#endif

#ifdef MAC_WITH_GPU
// The C++ drop-in layer of the device path; compiled in only for _ref/mac_ref_gpu.
#include "mac_gpu/Mac_GPU.h"
#endif

#include "solve3.h"
#include "state_format.h"

using namespace std;

// ---------------------------------------------------------------------------
// Linear-solver policy with the Policy_Solve_Linear_Umfpack member functions.
// ---------------------------------------------------------------------------
static double g_cg_rtol = 1e-14;
static long g_cg_iters_total = 0;
// When set, the assembled system (n, CSC arrays, right-hand side and solution) of
// every solve is appended to this file: lets the tests pin the CG stand-in
// against a sparse direct solve of the very arrays the reference assembled.
static FILE* g_csc_dump = nullptr;

class Policy_Solve_Linear_OracleCG {
  int m_n = 0;
  int* m_off = nullptr;
  int* m_ind = nullptr;
  double* m_val = nullptr;

 public:
  void Solve_Linear_FactorizeMatrice(int n, int* offset, int* indice, double* value) {
    m_n = n; m_off = offset; m_ind = indice; m_val = value;
  }
  static void dump(int n, const int* off, const int* ind, const double* val, const double* b, const double* x) {
    if (!g_csc_dump) return;
    int64_t nn = n, nnz = off[n];
    fwrite(&nn, 8, 1, g_csc_dump);
    fwrite(&nnz, 8, 1, g_csc_dump);
    fwrite(off, 4, n + 1, g_csc_dump);
    fwrite(ind, 4, nnz, g_csc_dump);
    fwrite(val, 8, nnz, g_csc_dump);
    fwrite(b, 8, n, g_csc_dump);
    fwrite(x, 8, n, g_csc_dump);
  }
  void Solve_Linear_Clean() { m_n = 0; }
  // Solves A x = b for the assembled (symmetric, negative definite) CSC matrix.
  void Solve_Linear(int n, int* off, int* ind, double* val, double* b, double* x) {
    std::vector<double> d(n, 0.0), r(n), z(n), p(n), q(n);
    for (int j = 0; j < n; ++j)
      for (int k = off[j]; k < off[j + 1]; ++k)
        if (ind[k] == j) d[j] = -val[k];
    double bn = 0;
    for (int i = 0; i < n; ++i) { x[i] = 0; r[i] = -b[i]; bn += b[i] * b[i]; }
    bn = sqrt(bn);
    if (bn == 0) { dump(n, off, ind, val, b, x); return; }
    double rz = 0;
    for (int i = 0; i < n; ++i) { z[i] = r[i] / d[i]; p[i] = z[i]; rz += r[i] * z[i]; }
    for (int it = 0; it < 100000; ++it) {
      std::fill(q.begin(), q.end(), 0.0);
      for (int j = 0; j < n; ++j)
        for (int k = off[j]; k < off[j + 1]; ++k) q[ind[k]] -= val[k] * p[j];
      double pq = 0;
      for (int i = 0; i < n; ++i) pq += p[i] * q[i];
      double a = rz / pq, rn = 0;
      for (int i = 0; i < n; ++i) { x[i] += a * p[i]; r[i] -= a * q[i]; rn += r[i] * r[i]; }
      ++g_cg_iters_total;
      if (sqrt(rn) <= g_cg_rtol * bn) break;
      double rz2 = 0;
      for (int i = 0; i < n; ++i) { z[i] = r[i] / d[i]; rz2 += r[i] * z[i]; }
      double beta = rz2 / rz;
      rz = rz2;
      for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
    dump(n, off, ind, val, b, x);
  }
};

// Linear-solver policy for the 3x3 corner systems of the boundary-condition
// extrapolation (the member functions of Policy_Solve_Linear_Umfpack, with its
// type_linear_solver typedef): the CSC matrix as a dense row-major array, solved
// by the checkers' shared Gaussian elimination (solve3.h).
class Policy_Solve_Linear_Dense3 {
  double m_a[9];

 public:
  typedef Policy_Solve_Linear_Dense3 type_linear_solver;
  void Solve_Linear_FactorizeMatrice(int n, int* off, int* ind, double* val) {
    for (int i = 0; i < 9; ++i) m_a[i] = 0.0;
    if (n != 3) return;
    for (int j = 0; j < 3; ++j)
      for (int k = off[j]; k < off[j + 1]; ++k) m_a[3 * ind[k] + j] = val[k];
  }
  void Solve_Linear(int n, int*, int*, double*, double* b, double* x) {
    if (n == 3) mac_solve3(m_a, b, x);
  }
  void Solve_Linear_Clean() {}
};

// Shared counter-based jitter (same function in the oracle and on the GPU).
static uint64_t g_refill_seed = 0;

template <typename Data>
class Policy_Add_Particle_Jitter8 {
  typedef typename Data::type_data_struct::type_Data_Grid type_Data_Grid;
  typedef typename type_Data_Grid::type_key type_key;
  typedef typename type_Data_Grid::type_spacing_vector type_spacing_vector;
  typedef typename Data::type_data_struct::type_Data_Topology type_Data_Topology;
  typedef typename type_Data_Topology::type_particle_list type_particle_list;
  typedef typename type_Data_Topology::type_particle type_particle;
  typedef typename type_particle::type_data_vector type_data_vector;
  type_particle_list& m_list;
  const type_spacing_vector& m_h;

 public:
  Policy_Add_Particle_Jitter8(const Data& data)
      : m_list(data.m_data.GetTopologyData().GetRefToParticleList()),
        m_h(data.m_data.GetGridData().m_h.GetRef()) {}
  void AddParticle(const type_key& k) {
    for (int s = 0; s < 8; ++s) {
      double pos[3];
      mac_jitter8_position(g_refill_seed, k.Get(1), k.Get(2), k.Get(3), s,
                           m_h.Get(1), m_h.Get(2), m_h.Get(3), pos);
      type_data_vector v;
      v.Set(1, pos[0]); v.Set(2, pos[1]); v.Set(3, pos[2]);
      m_list.push_back(type_particle(v));
    }
  }
};

// The refill policy named by the state header: Jitter8, or the reference's
// Policy_Add_Particle_Cube(n) for n >= 1.
template <typename Data>
class Policy_Add_Particle_Select {
  Policy_Add_Particle_Jitter8<Data> m_jitter;
  Policy_Add_Particle_Cube<Data> m_cube;
  int m_n;

 public:
  Policy_Add_Particle_Select(const Data& data, int n) : m_jitter(data), m_cube(data, n > 0 ? n : 1), m_n(n) {}
  template <typename Key>
  void AddParticle(const Key& k) {
    if (m_n > 0) m_cube.AddParticle(k);
    else m_jitter.AddParticle(k);
  }
};

// ---------------------------------------------------------------------------
// The world.
// ---------------------------------------------------------------------------
static int run(int argc, char** argv) {
  if (argc < 4) {
    fprintf(stderr,
            "usage: mac_ref <cmd> in.state out.state [n]\n"
            "  cmd: firstinit | step | topology | forces | ode | project | extrapolate | move | csc | bench\n");
    return 2;
  }
  std::string cmd = argv[1];
  mac_state_file st;
  if (mac_state_read(argv[2], &st) != 0) { fprintf(stderr, "cannot read %s\n", argv[2]); return 1; }
  int nrep = (argc > 4 && cmd != "csc") ? atoi(argv[4]) : 1;
  // The relative residual of the stand-in solve (1e-14 for parity work; the
  // throughput metric is quoted at 1e-8).
  if (const char* rt = getenv("MAC_REF_RTOL")) g_cg_rtol = atof(rt);

  const int DIM = 3;
  typedef double type_data_value;
  const int N = MAC_BRICK;
  const int NStock = N * N * N;
#ifdef MAC_PIPELINE_B
  const int NBSpeed = 3;  // Algorithms_RungeKutta_all needs 3 speeds (src/Algorithms_RungeKutta_all.h:6)
#else
  const int NBSpeed = 2;
#endif

  typedef Data_Base_Dim_Type<type_data_value, DIM> type_Data_Type;
  type_Data_Type m_data_type;
  typedef Data_Staggered_Left<type_Data_Type> type_Data_Base;
  type_Data_Base data_base(m_data_type);

#ifdef MAC_DEPTH
  typedef Data_CellType_Fluid_Air_Solid_Inflow_Interior_0_Pres<type_Data_Base> type_cell_type2;
#else
  typedef Data_CellType_Fluid_Air_Solid_Inflow<type_Data_Base> type_cell_type2;
#endif
  typedef Inversible_Value<type_data_value> type_inversible_value;
  type_inversible_value rho_air(1);
  type_inversible_value rho_fluid(1000);
  type_cell_type2 m_celltype2(data_base);
  m_celltype2.SetRhoAir(rho_air);
  m_celltype2.SetRhoFluid(rho_fluid);
#ifdef MAC_DEPTH
  typedef Data_CellType_Domain_Fluid_Without_0_Pres<type_cell_type2> type_cell_type;
#else
  typedef Data_CellType_Domain_Fluid<type_cell_type2> type_cell_type;
#endif
  type_cell_type m_celltype(m_celltype2);
  typedef Data_Grid_CellType_To_Grid_CellType<type_cell_type> type_cell_cell;
  type_cell_cell m_cell_cell(m_celltype);
  typedef typename type_cell_type2::Material_Type Mat;

  typedef bitset<DIM> type_const;
  type_const m_const;
  typedef Data_Grid_Speed<type_Data_Base, type_const> type_grid_speed;
  type_grid_speed m_grid_speed(m_const);
  for (int i = 1; i <= DIM; ++i) m_grid_speed.Set(i, 0.0, true);

  typedef Data_Grid_Pressure<type_Data_Base> type_grid_pressure;
  type_grid_pressure m_grid_pressure;
  m_grid_pressure.Pressure_Set(0.0);

  typedef Data_Grid_Layer<int> type_layer2;
  type_layer2 m_layer2(-1);
  typedef Data_Grid_Layer_Empty<type_layer2> type_layer;
  type_layer m_layer(m_layer2);
  typedef Data_Grid_Layer<int> type_id2;
  type_id2 m_id2(-1);
  typedef Data_Grid_Layer_Empty<type_id2> type_id;
  type_id m_id(m_id2);

  typedef Data_Chunk_Layer<type_layer, NStock> type_chunk_layer;
  type_chunk_layer m_chunk_layer(m_layer);
  typedef Data_Chunk_Id_Cell<type_id, NStock> type_chunk_id;
  type_chunk_id m_chunk_id(m_id);
  typedef Data_Chunk_Bool_Array<NStock> type_bool_array;
  type_bool_array m_bool_array;
  typedef Data_Chunk_CellType<type_cell_cell, NStock> type_chunk_celltype;
  type_chunk_celltype m_chunk_celltype(m_cell_cell);
  typedef Data_Chunk_Speed<type_grid_speed, NBSpeed, 1, NStock> type_chunk_speed;
  type_chunk_speed m_chunk_speed(m_grid_speed);
  typedef Data_Chunk_Pressure<type_grid_pressure, NStock> type_chunk_pressure;
  type_chunk_pressure m_chunk_pressure(m_grid_pressure);
#ifdef MAC_DEPTH
  typedef Data_Grid_Depth<int> type_depth2;
  type_depth2 m_depth2(-1);
  typedef Data_Grid_Depth_Empty<type_depth2> type_depth;
  type_depth m_depth(m_depth2);
  typedef Data_Chunk_Depth<type_depth, NStock> type_chunk_depth;
  type_chunk_depth m_chunk_depth(m_depth);
  typedef Data_Chunk<type_bool_array, type_chunk_layer, type_chunk_depth, type_chunk_id, type_chunk_celltype, type_chunk_speed, type_chunk_pressure> type_chunk;
  type_chunk m_chunk(m_bool_array, m_chunk_layer, m_chunk_depth, m_chunk_id, m_chunk_celltype, m_chunk_speed, m_chunk_pressure);
#else
  typedef Data_Chunk<type_bool_array, type_chunk_layer, type_chunk_id, type_chunk_celltype, type_chunk_speed, type_chunk_pressure> type_chunk;
  type_chunk m_chunk(m_bool_array, m_chunk_layer, m_chunk_id, m_chunk_celltype, m_chunk_speed, m_chunk_pressure);
#endif
  typedef Neighbour_List_Empty<DIM, type_chunk> type_neigh;
  type_neigh m_neigh(m_chunk);

  typedef Offset<int, DIM, N> type_off;
  typedef Offset_Base<type_off, type_neigh> type_off_base;
  typedef Offset_Base_Layer<type_layer, type_off_base> type_off_base_layer;
#ifdef MAC_DEPTH
  typedef Offset_Base_Depth<type_depth, type_off_base_layer> type_off_base_depth;
  typedef Offset_Base_Id_Cell<type_id, type_off_base_depth> type_off_base_id;
#else
  typedef Offset_Base_Id_Cell<type_id, type_off_base_layer> type_off_base_id;
#endif
  typedef Offset_Base_CellType<type_cell_cell, type_off_base_id> type_off_base_celltype;
  typedef Offset_Base_Speed<type_grid_speed, type_off_base_celltype> type_off_base_speed;
  typedef Offset_Base_Pressure<type_grid_pressure, type_off_base_speed> type_off_base_pressure;
  typedef Offset_Base_Neighbour<type_off_base_pressure> type_off_base_neighbour;
  typedef Physvector<DIM, int> vect;
  typedef HashPhysvector<DIM, int> Hash;
  Hash hash;
  typedef ChunkHashTable<Hook_Neighbour_List_Chunk, vect, type_neigh, type_off_base_neighbour, Hash> type_chunk_table;
  type_chunk_table m_chunk_table(m_neigh, hash);

  typedef Data_Viscosity<type_chunk_table> type_data_viscosity;
  type_data_viscosity m_data_viscosity(m_chunk_table);
  m_data_viscosity.m_viscosity = st.hdr.viscosity;
  typedef Data_Grid_Base_Spacing<type_data_viscosity, Physvector<DIM, type_data_value>> type_data_grid;
  type_data_grid m_data_grid(m_data_viscosity);
  Physvector<DIM, type_data_value> h;
  h.Set(1, st.hdr.h[0]); h.Set(2, st.hdr.h[1]); h.Set(3, st.hdr.h[2]);
  m_data_grid.m_h.Set(h);
  typedef Data_Staggered_Left<type_data_grid> type_stag_left;
  type_stag_left m_stag_left(m_data_grid);
  typedef Data_CellType_Interface_Constant<type_stag_left> type_interface_constant;
  type_interface_constant m_type_interface_constant(m_stag_left);
  typedef Data_Grid_Data<type_interface_constant, type_Data_Base> type_grid_data;
  type_grid_data m_grid_data(m_type_interface_constant, data_base);

#ifdef MAC_PIPELINE_B
  typedef Data_Particle<type_Data_Base, 3> type_particle;  // pos0..pos2 of the RK4 over particles
#else
  typedef Data_Particle<type_Data_Base> type_particle;
#endif
  typedef Data_Particles_List<type_particle, type_Data_Base> type_particles;
  type_particles particles(data_base);
  typedef Data_Topology<type_particles, type_grid_data> type_topology;
  type_topology m_topology(particles, m_grid_data);

  typedef Data_Timing_Time<type_data_value> type_time;
  type_time m_time;
  m_time.m_t = st.hdr.t;
  m_time.m_dt = st.hdr.dt;
  m_time.m_factor = st.hdr.cfl_factor;
  typedef Data_Timing<type_time, type_topology> type_timing;
  type_timing m_timing(m_time, m_topology);
  typedef DataRef<type_timing> type_data_ref;
  type_data_ref m_data_ref(m_timing);
  auto& grid = m_data_ref.m_data.GetGridData();
  auto& plist = m_data_ref.m_data.GetTopologyData().GetRefToParticleList();
  auto& timing = m_data_ref.m_data.GetTimingData();
  g_refill_seed = st.hdr.step;

  // ---- load ----
  for (int64_t c = 0; c < st.hdr.nchunks; ++c) {
    const int32_t* ck = st.keys + 3 * c;
    vect k0;
    k0.Set(1, ck[0] * N); k0.Set(2, ck[1] * N); k0.Set(3, ck[2] * N);
    grid[k0];
    vect ckey;
    ckey.Set(1, ck[0]); ckey.Set(2, ck[1]); ckey.Set(3, ck[2]);
    type_chunk& ch = grid.DirectAcessChunk(ckey);
    for (int o = 0; o < NStock; ++o) {
      size_t idx = (size_t)c * NStock + o;
      ch.GetChunk_Bool_Array()[o] = st.exists[idx] != 0;
      for (int b = 0; b < 2; ++b) {
        type_grid_speed& s = ch.Speed_GetPointer(b)[o];
        for (int i = 1; i <= 3; ++i) s.m_speed.Set(i, st.u[b][i - 1][idx]);
      }
      type_grid_speed& a = ch.Acceleration_GetPointer(0)[o];
      for (int i = 1; i <= 3; ++i) a.m_speed.Set(i, st.acc[i - 1][idx]);
      type_grid_speed& s0 = ch.Speed_GetPointer(0)[o];
      for (int i = 1; i <= 3; ++i) {
        if (st.flags[idx] & (1u << (i - 1))) s0.Set_Const(i); else s0.Set_None_Const(i);
      }
      ch.Pressure_GetPointer()[o].Pressure_Set(st.p[idx]);
      type_cell_cell& ct = ch.CellType_GetPointer()[o];
      switch (st.type[idx]) {
        case MAC_AIR: ct.m_mat = Mat::Air; break;
        case MAC_FLUID: ct.m_mat = Mat::Fluid; break;
        case MAC_SOLID: ct.m_mat = Mat::Solid; break;
#ifdef MAC_DEPTH
        case MAC_INTERIOR: ct.m_mat = Mat::Interior; break;
#endif
        default: ct.m_mat = Mat::Inflow; break;
      }
#ifdef MAC_DEPTH
      ch.Depth_GetPointer()[o].SetDepth(st.depth[idx]);
#endif
      ct.SetIsNoDelete((st.flags[idx] & MAC_FLAG_NODELETE) != 0);
      ch.Layer_GetPointer()[o].SetLayer(st.layer[idx]);
      ch.Id_Cell_GetPointer()[o].SetLayer(st.id[idx]);
    }
  }
  for (int64_t q = 0; q < st.hdr.nparticles; ++q) {
    Physvector<DIM, double> v;
    v.Set(1, st.pos[3 * q]); v.Set(2, st.pos[3 * q + 1]); v.Set(3, st.pos[3 * q + 2]);
    plist.push_back(type_particle(v));
  }

  // ---- policies and algorithms (test/TestJetDEau_Basic.cpp:287-432) ----
  typedef Policies<> type_pol_empty;
  type_pol_empty m_pol_empty;
  typedef Algorithms_Speed_Constant_Mirror<type_data_ref, type_pol_empty> type_alg_mirror;
  type_alg_mirror m_alg_mirror(m_data_ref, m_pol_empty);
  typedef Algorithms_Solid_To_Const<type_data_ref, type_pol_empty> type_alg_solid;
  type_alg_solid m_alg_solid(m_data_ref, m_pol_empty);
  typedef Algorithms_Extrapolate<type_data_ref, type_pol_empty> type_alg_extrapolate;
  type_alg_extrapolate m_alg_extrapolate(m_data_ref, m_pol_empty);
  // Algorithm_Extrapolate_Boundary_Condition (3D form) with the policies of
  // test/Lateral_jet_3.cpp:491-498 that it reads: Policy_Is_In_Domain_Speed
  // and the linear solver (here the dense 3x3 policy above).
  typedef Policy_Is_In_Domain_Speed<type_data_ref> type_pol_in_domain_speed;
  type_pol_in_domain_speed m_pol_in_domain_speed;
  Policy_Solve_Linear_Dense3 m_pol_dense3;
  typedef Policies<type_pol_in_domain_speed, Policy_Solve_Linear_Dense3> type_pol_extrap_bc;
  type_pol_extrap_bc m_pol_extrap_bc(m_pol_in_domain_speed, m_pol_dense3);
  typedef Algorithm_Extrapolate_Boundary_Condition<type_data_ref, type_pol_extrap_bc> type_alg_extrap_bc;
  type_alg_extrap_bc m_alg_extrap_bc(m_data_ref, m_pol_extrap_bc);

  typedef Policy_Layer_Max<type_data_ref> type_pol_layer;
  type_pol_layer m_pol_layer(st.hdr.layer_max);
  typedef Policy_Particle_To_Key<type_data_ref> type_pol_part_to_key;
  type_pol_part_to_key m_pol_part_to_key(m_data_ref);
  typedef Policy_CheckDT<type_data_ref> type_pol_check_dt;
  type_pol_check_dt m_pol_check_dt(st.hdr.dt_min, st.hdr.dt_max);
  typedef Policy_Add_Particle_Select<type_data_ref> type_pol_add_particle;
  type_pol_add_particle m_add_particle(m_data_ref, st.hdr.refill_cube);
  typedef Policy_Is_Inbound_Filling_Layer_CellType<type_data_ref> type_pol_fill;
  type_pol_fill m_pol_fill;
#ifdef MAC_DEPTH
  typedef Policy_Depth<type_data_ref> type_pol_depth;
  type_pol_depth m_pol_depth(st.hdr.depth_max, st.hdr.depth_interior, st.hdr.depth_remove);
  typedef Policies<type_pol_layer, type_pol_part_to_key, type_pol_check_dt, type_pol_add_particle, type_pol_fill, type_pol_depth> type_pol_init;
  type_pol_init m_pol_init(m_pol_layer, m_pol_part_to_key, m_pol_check_dt, m_add_particle, m_pol_fill, m_pol_depth);
#else
  typedef Policies<type_pol_layer, type_pol_part_to_key, type_pol_check_dt, type_pol_add_particle, type_pol_fill> type_pol_init;
  type_pol_init m_pol_init(m_pol_layer, m_pol_part_to_key, m_pol_check_dt, m_add_particle, m_pol_fill);
#endif

#ifdef MAC_DEPTH
  typedef Algorithms_Initialize_Layer_And_Depth<type_data_ref, type_pol_init> type_alg_initialize_mac;
#else
  typedef Algorithms_Initialize_MacCell<type_data_ref, type_pol_init> type_alg_initialize_mac;
#endif
  type_alg_initialize_mac m_alg_initialize_mac(m_data_ref, m_pol_init);
#ifdef MAC_DEPTH
  typedef Algorithms_Create_Fluid_Particle_Depth<type_data_ref, type_pol_init> type_alg_create;
#else
  typedef Algorithms_Create_Fluid_Particle<type_data_ref, type_pol_init> type_alg_create;
#endif
  type_alg_create m_alg_create(m_data_ref, m_pol_init);
#ifdef MAC_DEPTH
  typedef Algorithms_Layer_Initial_With_Particle_Depth<type_data_ref, type_pol_init> type_alg_layer_initial;
#else
  typedef Algorithms_Layer_Initial_With_Particle<type_data_ref, type_pol_init> type_alg_layer_initial;
#endif
  type_alg_layer_initial m_alg_layer_initial(m_data_ref, m_pol_init);
#ifdef MAC_DEPTH
  typedef Algorithms_Update_CellType_Layer_Depth<type_data_ref, type_pol_init> type_alg_update_celltype;
#else
  typedef Algorithms_Update_CellType_Layer<type_data_ref, type_pol_init> type_alg_update_celltype;
#endif
  type_alg_update_celltype m_alg_update_celltype(m_data_ref, m_pol_init);
  typedef Algorithms_Delete_MacCell<type_data_ref, type_pol_init> type_alg_delete;
  type_alg_delete m_alg_delete(m_data_ref, m_pol_init);
  typedef Algorithms_Calculate_Time_Step<type_data_ref, type_pol_init> type_alg_dt;
  type_alg_dt m_alg_dt(m_data_ref, m_pol_init);

  typedef Algorithms<type_alg_initialize_mac, type_alg_layer_initial, type_alg_create, type_alg_update_celltype, type_alg_delete, type_alg_dt> type_alg_init;
  type_alg_init m_alg_init(m_alg_initialize_mac, m_alg_layer_initial, m_alg_create, m_alg_update_celltype, m_alg_delete, m_alg_dt);
  typedef Algorithms<type_alg_solid, type_alg_mirror, type_alg_initialize_mac, type_alg_create, type_alg_layer_initial, type_alg_update_celltype, type_alg_delete, type_alg_extrapolate> type_alg_first_init;
  type_alg_first_init m_alg_first_init(m_alg_solid, m_alg_mirror, m_alg_initialize_mac, m_alg_create, m_alg_layer_initial, m_alg_update_celltype, m_alg_delete, m_alg_extrapolate);

  typedef Policy_Gravity<type_data_ref> type_pol_gravity;
  type_pol_gravity m_pol_gravity(m_data_ref, st.hdr.gravity, st.hdr.gravity_axis);
  typedef Policy_Speed_Interpolation_Linear_Symmetric<type_data_ref> type_pol_interp_sym;
  type_pol_interp_sym m_pol_interp_sym(m_data_ref);
  typedef Policy_Convection_Apply_If<type_data_ref> type_pol_conv_if;
  type_pol_conv_if m_pol_conv_if;
  typedef Policy_Upwind_1_Order<type_data_ref, type_pol_interp_sym> type_pol_conv;
  type_pol_conv m_pol_conv(m_data_ref, m_pol_interp_sym);
  typedef Policies<type_pol_gravity, type_pol_conv_if, type_pol_conv> type_pol_grid;
  type_pol_grid m_pol_grid(m_pol_gravity, m_pol_conv_if, m_pol_conv);
  typedef Algorithms_Gravity<type_data_ref, type_pol_grid> type_alg_gravity;
  type_alg_gravity m_alg_gravity(m_data_ref, m_pol_grid);
  typedef Algorithms_Convection<type_data_ref, type_pol_grid> type_alg_convection;
  type_alg_convection m_alg_convection(m_data_ref, m_pol_grid);
  typedef Algorithms<type_alg_gravity, type_alg_convection> type_alg_solve_grid;
  type_alg_solve_grid m_alg_solve_grid(m_alg_gravity, m_alg_convection);

  typedef Policy_Solve_Linear_OracleCG type_pol_solve_linear;
  type_pol_solve_linear m_pol_solve_linear;
  typedef Policy_Divergence<type_data_ref> type_pol_divergence;
  type_pol_divergence m_pol_divergence(m_data_ref);
  typedef Policy_Gradiant<type_data_ref> type_pol_gradiant;
  type_pol_gradiant m_pol_gradiant(m_data_ref);
  typedef Policy_Von_Neumann_Boundary<type_data_ref> type_pol_vn;
  type_pol_vn m_pol_vn(m_data_ref);
  typedef Policy_Pressure_If_Correction<type_data_ref> type_pol_pres_if;
  type_pol_pres_if m_pol_pres_if;
  typedef Policies<type_pol_solve_linear, type_pol_divergence, type_pol_gradiant, type_pol_vn, type_pol_pres_if> type_pol_pres;
  type_pol_pres m_pol_pres(m_pol_solve_linear, m_pol_divergence, m_pol_gradiant, m_pol_vn, m_pol_pres_if);
  typedef Algorithms_Solve_Pressure<type_data_ref, type_pol_pres> type_alg_solve_pressure;
  type_alg_solve_pressure m_alg_solve_pressure(m_data_ref, m_pol_pres);
  typedef Algorithms_Do_Pressure<type_data_ref, type_alg_solve_pressure> type_alg_do_pressure;
  type_alg_do_pressure m_alg_do_pressure(m_data_ref, m_alg_solve_pressure);

  typedef Policies<type_alg_solve_grid, type_alg_solve_pressure> type_pol_ODE;
  type_pol_ODE m_pol_ODE(m_alg_solve_grid, m_alg_solve_pressure);
  typedef Algorithms_RungeKutta_RK2_TVD<type_data_ref, type_pol_ODE> type_alg_ODE;
  type_alg_ODE m_alg_ODE(m_data_ref, m_pol_ODE);

  // viscous composition (test/Lateral_jet_3.cpp:533-605 with VISCOSITY)
  typedef Policy_Laplacian_Speed<type_data_ref> type_pol_lap_speed;
  type_pol_lap_speed m_pol_lap_speed(m_data_ref);
  typedef Policy_Viscosity_Apply_If<type_data_ref> type_pol_visc_if;
  type_pol_visc_if m_pol_visc_if;
  typedef Policies<type_pol_gravity, type_pol_conv_if, type_pol_conv, type_pol_lap_speed, type_pol_visc_if> type_pol_grid_v;
  type_pol_grid_v m_pol_grid_v(m_pol_gravity, m_pol_conv_if, m_pol_conv, m_pol_lap_speed, m_pol_visc_if);
  typedef Algorithms_Viscosity<type_data_ref, type_pol_grid_v> type_alg_viscosity;
  type_alg_viscosity m_alg_viscosity(m_data_ref, m_pol_grid_v);
  typedef Algorithms<type_alg_gravity, type_alg_convection, type_alg_viscosity> type_alg_solve_grid_v;
  type_alg_solve_grid_v m_alg_solve_grid_v(m_alg_gravity, m_alg_convection, m_alg_viscosity);
  typedef Policy_Dirichlet_Boundary<type_data_ref> type_pol_dirichlet;
  type_pol_dirichlet m_pol_dirichlet(m_data_ref);
  typedef Policies<type_pol_solve_linear, type_pol_divergence, type_pol_gradiant, type_pol_vn, type_pol_pres_if, type_pol_dirichlet> type_pol_pres_v;
  type_pol_pres_v m_pol_pres_v(m_pol_solve_linear, m_pol_divergence, m_pol_gradiant, m_pol_vn, m_pol_pres_if, m_pol_dirichlet);
  typedef Algorithms_Solve_Pressure_Dirichlet<type_data_ref, type_pol_pres_v> type_alg_solve_pressure_v;
  type_alg_solve_pressure_v m_alg_solve_pressure_v(m_data_ref, m_pol_pres_v);
  typedef Algorithms_Do_Pressure<type_data_ref, type_alg_solve_pressure_v> type_alg_do_pressure_v;
  type_alg_do_pressure_v m_alg_do_pressure_v(m_data_ref, m_alg_solve_pressure_v);
  typedef Policies<type_alg_solve_grid_v, type_alg_solve_pressure_v> type_pol_ODE_v;
  type_pol_ODE_v m_pol_ODE_v(m_alg_solve_grid_v, m_alg_solve_pressure_v);
  typedef Algorithms_RungeKutta_RK2_TVD<type_data_ref, type_pol_ODE_v> type_alg_ODE_v;
  type_alg_ODE_v m_alg_ODE_v(m_data_ref, m_pol_ODE_v);

#ifdef MAC_PIPELINE_B
  // Pipeline B, test/Jet3.cpp:546-675 (no SPLIT, VISCOSITY): the per-step init
  // with dt and the extrapolation, then Algorithms_RungeKutta_all over
  // Policies<Algorithms<solve_grid, force projection, extrapolation of the
  // acceleration>, Policy_Move_Particle>, where solve_grid re-runs the topology
  // (with Create_Interior_Depth) at every stage before gravity, convection and
  // viscosity. Deviations: the Dirichlet projection solves with the stand-in
  // policy instead of pyamg (Algorithmes_Solve_Pressure_Dirichlet_Pyamg.h
  // assembles the same system with the opposite sign), and
  // Algorithm_Extrapolate_Boundary_Condition is left out of both
  // extrapolations (its result depends on the hash map's visiting order).
  typedef Algorithms_Create_Interior_Depth<type_data_ref, type_pol_init> type_alg_create_interior;
  type_alg_create_interior m_alg_create_interior(m_data_ref, m_pol_init);
  typedef Algorithms<type_alg_initialize_mac, type_alg_layer_initial, type_alg_create, type_alg_update_celltype, type_alg_delete, type_alg_dt, type_alg_extrapolate> type_alg_init_b;
  type_alg_init_b m_alg_init_b(m_alg_initialize_mac, m_alg_layer_initial, m_alg_create, m_alg_update_celltype, m_alg_delete, m_alg_dt, m_alg_extrapolate);
  typedef Algorithms<type_alg_initialize_mac, type_alg_layer_initial, type_alg_create_interior, type_alg_update_celltype, type_alg_delete, type_alg_extrapolate> type_alg_init2;
  type_alg_init2 m_alg_init2(m_alg_initialize_mac, m_alg_layer_initial, m_alg_create_interior, m_alg_update_celltype, m_alg_delete, m_alg_extrapolate);
  typedef Algorithms<type_alg_init2, type_alg_gravity, type_alg_convection, type_alg_viscosity> type_alg_solve_grid_b;
  type_alg_solve_grid_b m_alg_solve_grid_b(m_alg_init2, m_alg_gravity, m_alg_convection, m_alg_viscosity);
  typedef Algorithms_Solve_Pressure_Force<type_data_ref, type_alg_solve_pressure_v> type_alg_force_pressure;
  type_alg_force_pressure m_alg_force_pressure(m_data_ref, m_alg_solve_pressure_v);
  typedef Algorithms<type_alg_extrapolate> type_alg_extrap_only;
  type_alg_extrap_only m_alg_extrap_only(m_alg_extrapolate);
  typedef Algorithms_Accel_To_Speed<type_data_ref, type_alg_extrap_only> type_alg_extrap_force;
  type_alg_extrap_force m_alg_extrap_force(m_data_ref, m_alg_extrap_only);
  typedef Algorithms<type_alg_solve_grid_b, type_alg_force_pressure, type_alg_extrap_force> type_alg_solve_grid_force;
  type_alg_solve_grid_force m_alg_solve_grid_force(m_alg_solve_grid_b, m_alg_force_pressure, m_alg_extrap_force);
  typedef Policies<type_pol_interp_sym> type_pol_move_b;
  type_pol_move_b m_pol_move_b(m_pol_interp_sym);
  typedef Policy_Move_Particle<type_data_ref, type_pol_move_b> type_pol_move2;
  type_pol_move2 m_pol_move2(m_data_ref, m_pol_move_b);
  typedef Policies<type_alg_solve_grid_force, type_pol_move2> type_pol_ODE_b;
  type_pol_ODE_b m_pol_ODE_b(m_alg_solve_grid_force, m_pol_move2);
  typedef Algorithms_RungeKutta_all<type_data_ref, type_pol_ODE_b> type_alg_ODE_b;
  type_alg_ODE_b m_alg_ODE_b(m_data_ref, m_pol_ODE_b);
#endif

  typedef Policy_Advance_Ode_RungeKutta<type_data_ref> type_pol_advance;
  type_pol_advance m_pol_advance;
  typedef Policies<type_pol_advance, type_pol_interp_sym> type_pol_move;
  type_pol_move m_pol_move(m_pol_advance, m_pol_interp_sym);
  typedef Algorithms_Move_Particles<type_data_ref, type_pol_move> type_alg_move;
  type_alg_move m_alg_move(m_data_ref, m_pol_move);
  typedef Policy_Speed_Interpolation_Linear<type_data_ref> type_pol_interp_lin;
  type_pol_interp_lin m_pol_interp_lin(m_data_ref);
  typedef Policies<type_pol_advance, type_pol_interp_lin> type_pol_move_lin;
  type_pol_move_lin m_pol_move_lin(m_pol_advance, m_pol_interp_lin);
  typedef Algorithms_Move_Particles<type_data_ref, type_pol_move_lin> type_alg_move_lin;
  type_alg_move_lin m_alg_move_lin(m_data_ref, m_pol_move_lin);

#ifdef MAC_WITH_GPU
  // The same world driven through the drop-in layer: the unmodified
  // Algorithms_Solve_Pressure with Policy_Solve_Linear_GPU as its solver policy,
  // and the pipeline-A step as device algorithms.
  typedef Policies<Policy_Solve_Linear_GPU, type_pol_divergence, type_pol_gradiant, type_pol_vn, type_pol_pres_if> type_pol_pres_gpu;
  Policy_Solve_Linear_GPU m_pol_solve_gpu(g_cg_rtol);
  type_pol_pres_gpu m_pol_pres_gpu(m_pol_solve_gpu, m_pol_divergence, m_pol_gradiant, m_pol_vn, m_pol_pres_if);
  typedef Algorithms_Solve_Pressure<type_data_ref, type_pol_pres_gpu> type_alg_solve_pressure_gpu;
  type_alg_solve_pressure_gpu m_alg_solve_pressure_gpu(m_data_ref, m_pol_pres_gpu);
  typedef Algorithms_Do_Pressure<type_data_ref, type_alg_solve_pressure_gpu> type_alg_do_pressure_gpu;
  type_alg_do_pressure_gpu m_alg_do_pressure_gpu(m_data_ref, m_alg_solve_pressure_gpu);

  mac_params gprm;
  mac_default_params(&gprm);
  for (int i = 0; i < 3; ++i) gprm.h[i] = st.hdr.h[i];
  gprm.cfl_factor = st.hdr.cfl_factor;
  gprm.dt_min = st.hdr.dt_min;
  gprm.dt_max = st.hdr.dt_max;
  gprm.gravity = st.hdr.gravity;
  gprm.gravity_axis = st.hdr.gravity_axis;
  gprm.layer_max = st.hdr.layer_max;
  gprm.interp_symmetric = st.hdr.interp_symmetric;
  gprm.viscosity = st.hdr.viscosity;
  gprm.depth_mode = st.hdr.depth_mode;
  gprm.depth_max = st.hdr.depth_max;
  gprm.depth_interior = st.hdr.depth_interior;
  gprm.depth_remove = st.hdr.depth_remove;
  gprm.refill_cube = st.hdr.refill_cube;
#ifdef MAC_PIPELINE_B
  gprm.pipeline = 1;  // Algorithms_Step_GPU runs the pipeline-B step of this world
#endif
  gprm.rtol = g_cg_rtol;
  gprm.max_iters = 5000;
  gprm.max_bricks = 8192;
  gprm.max_particles = 1 << 22;
  typedef Policy_Mac_GPU<type_data_ref> type_pol_gpu;
  type_pol_gpu m_pol_gpu(m_data_ref, gprm, g_refill_seed);
  Algorithms_Step_GPU<type_data_ref, type_pol_gpu> m_alg_step_gpu(m_data_ref, m_pol_gpu);
  Algorithms_To_Host_GPU<type_data_ref, type_pol_gpu> m_alg_to_host_gpu(m_data_ref, m_pol_gpu);

  // The reference's own RK2-TVD and Algorithms_Do_Pressure with the device
  // projection at the composable interface (Init_Iteration,
  // Divergence_Projection, End_Iteration): the host loops over the speed
  // buffers stay the reference's, only the projections run on the device.
  type_pol_gpu m_pol_gpu_proj(m_data_ref, gprm, g_refill_seed);
  typedef Algorithms_Solve_Pressure_GPU<type_data_ref, type_pol_gpu> type_alg_solve_pressure_dev;
  type_alg_solve_pressure_dev m_alg_solve_pressure_dev(m_data_ref, m_pol_gpu_proj);
  typedef Policies<type_alg_solve_grid, type_alg_solve_pressure_dev> type_pol_ODE_dev;
  type_pol_ODE_dev m_pol_ODE_dev(m_alg_solve_grid, m_alg_solve_pressure_dev);
  typedef Algorithms_RungeKutta_RK2_TVD<type_data_ref, type_pol_ODE_dev> type_alg_ODE_dev;
  type_alg_ODE_dev m_alg_ODE_dev(m_data_ref, m_pol_ODE_dev);
  typedef Algorithms_Do_Pressure<type_data_ref, type_alg_solve_pressure_dev> type_alg_do_pressure_dev;
  type_alg_do_pressure_dev m_alg_do_pressure_dev(m_data_ref, m_alg_solve_pressure_dev);
#endif

  // The reference algorithms print timing lines on std::cout; keep them out of the way.
  std::ofstream devnull("/dev/null");
  std::streambuf* saved = std::cout.rdbuf(devnull.rdbuf());

  auto fluid_count = [&]() {
    long n = 0;
    for (auto it = grid.begin(); it != grid.end(); ++it)
      if (it.data().CellType_GetRef().GetIsFluid()) ++n;
    return n;
  };

  long fluid_cell_steps = 0;
  auto t0 = std::chrono::steady_clock::now();
  for (int r = 0; r < nrep; ++r) {
    if (cmd == "firstinit") {
      m_alg_first_init.Do();
    } else if (cmd == "setup") {
      m_alg_solid.Do();
      m_alg_mirror.Do();
    } else if (cmd == "step" || cmd == "bench") {
      ++g_refill_seed;
      m_alg_init.Do();
      m_alg_ODE.Do();
      m_alg_extrapolate.Do();
      m_alg_move.Do();
      timing.m_t += timing.m_dt;
      if (cmd == "bench") fluid_cell_steps += fluid_count();
    } else if (cmd == "topology") {
      ++g_refill_seed;
      m_alg_init.Do();
    } else if (cmd == "forces") {
      type_chunk_speed::ispeed = 0;
      for (auto it = grid.begin(); it != grid.end(); ++it) it.data().Acceleration_GetRef().SetZero(true);
      m_alg_solve_grid.Do();
    } else if (cmd == "ode") {
      m_alg_ODE.Do();
    } else if (cmd == "project") {
      type_chunk_speed::ispeed = 0;
      m_alg_do_pressure.Do();
    } else if (cmd == "extrapolate") {
      m_alg_extrapolate.Do();
    } else if (cmd == "extrapbc") {
      type_chunk_speed::ispeed = 0;
      m_alg_extrap_bc.Do();
    } else if (cmd == "move") {
      m_alg_move.Do();
    } else if (cmd == "movelin") {
      m_alg_move_lin.Do();
#ifdef MAC_WITH_GPU
    } else if (cmd == "gpuproject") {
      type_chunk_speed::ispeed = 0;
      m_alg_do_pressure_gpu.Do();
    } else if (cmd == "gpuode") {
      m_alg_ODE_dev.Do();
      if (m_pol_gpu_proj.Session().Status() != MAC_OK) {
        std::cout.rdbuf(saved);
        fprintf(stderr, "device projection failed: %s\n", mac_error_string(m_pol_gpu_proj.Session().Status()));
        return 1;
      }
    } else if (cmd == "gpudopressure") {
      type_chunk_speed::ispeed = 0;
      m_alg_do_pressure_dev.Do();
      if (m_pol_gpu_proj.Session().Status() != MAC_OK) {
        std::cout.rdbuf(saved);
        fprintf(stderr, "device projection failed: %s\n", mac_error_string(m_pol_gpu_proj.Session().Status()));
        return 1;
      }
    } else if (cmd == "gpustep") {
      m_alg_step_gpu.Do();
      if (r + 1 == nrep) {
        m_alg_to_host_gpu.Do();
        g_refill_seed = m_pol_gpu.Session().Step();
        if (m_pol_gpu.Session().Status() != MAC_OK) {
          std::cout.rdbuf(saved);
          fprintf(stderr, "device step failed: %s\n", mac_error_string(m_pol_gpu.Session().Status()));
          return 1;
        }
      }
#endif
    } else if (cmd == "vforces") {
      type_chunk_speed::ispeed = 0;
      for (auto it = grid.begin(); it != grid.end(); ++it) it.data().Acceleration_GetRef().SetZero(true);
      m_alg_solve_grid_v.Do();
    } else if (cmd == "vproject") {
      type_chunk_speed::ispeed = 0;
      m_alg_do_pressure_v.Do();
    } else if (cmd == "vode") {
      m_alg_ODE_v.Do();
#ifdef MAC_PIPELINE_B
    } else if (cmd == "bstep") {
      ++g_refill_seed;
      m_alg_init_b.Do();
      m_alg_ODE_b.Do();
    } else if (cmd == "binit") {
      ++g_refill_seed;
      m_alg_init_b.Do();
    } else if (cmd == "bode") {
      m_alg_ODE_b.Do();
#endif
    } else if (cmd == "vstep") {
      ++g_refill_seed;
      m_alg_init.Do();
      m_alg_ODE_v.Do();
      m_alg_extrapolate.Do();
      m_alg_move.Do();
      timing.m_t += timing.m_dt;
    } else if (cmd == "csc") {
      // Projection of speed 0 with the assembled system written to argv[4].
      g_csc_dump = fopen(argv[4], "wb");
      type_chunk_speed::ispeed = 0;
      m_alg_do_pressure.Do();
      fclose(g_csc_dump);
      g_csc_dump = nullptr;
      break;
    } else {
      std::cout.rdbuf(saved);
      fprintf(stderr, "unknown command %s\n", cmd.c_str());
      return 2;
    }
  }
  auto t1 = std::chrono::steady_clock::now();
  std::cout.rdbuf(saved);
  double secs = std::chrono::duration<double>(t1 - t0).count();
  if (cmd == "bench") {
    printf("{\"fluid_cell_steps\": %ld, \"seconds\": %.6f, \"cg_iters\": %ld}\n", fluid_cell_steps, secs, g_cg_iters_total);
  }

  // ---- dump ----
  std::set<std::tuple<int, int, int>> cks;
  for (auto it = grid.begin(); it != grid.end(); ++it) {
    vect k = it.key();
    int c[3];
    for (int i = 0; i < 3; ++i) {
      int v = k.Get(i + 1);
      c[i] = v >= 0 ? v / N : (v + 1) / N - 1;
    }
    cks.insert(std::make_tuple(c[2], c[1], c[0]));
  }
  mac_state_file out;
  mac_state_alloc(&out, (int64_t)cks.size(), (int64_t)plist.size());
  out.hdr = st.hdr;
  out.hdr.nchunks = (int64_t)cks.size();
  out.hdr.nparticles = (int64_t)plist.size();
  out.hdr.t = timing.m_t;
  out.hdr.dt = timing.m_dt;
  out.hdr.step = g_refill_seed;
  int64_t c = 0;
  for (auto& t : cks) {
    vect ckey;
    ckey.Set(1, std::get<2>(t)); ckey.Set(2, std::get<1>(t)); ckey.Set(3, std::get<0>(t));
    out.keys[3 * c] = std::get<2>(t); out.keys[3 * c + 1] = std::get<1>(t); out.keys[3 * c + 2] = std::get<0>(t);
    type_chunk& ch = grid.DirectAcessChunk(ckey);
    for (int o = 0; o < NStock; ++o) {
      size_t idx = (size_t)c * NStock + o;
      out.exists[idx] = ch.GetChunk_Bool_Array()[o] ? 1 : 0;
      for (int b = 0; b < 2; ++b)
        for (int i = 1; i <= 3; ++i) out.u[b][i - 1][idx] = ch.Speed_GetPointer(b)[o].Get(i);
      for (int i = 1; i <= 3; ++i) out.acc[i - 1][idx] = ch.Acceleration_GetPointer(0)[o].Get(i);
      out.p[idx] = ch.Pressure_GetPointer()[o].Pressure_Get().Get();
      const type_grid_speed& s0 = ch.Speed_GetPointer(0)[o];
      uint8_t f = 0;
      for (int i = 1; i <= 3; ++i) if (s0.Get_Const(i)) f |= (uint8_t)(1u << (i - 1));
      type_cell_cell& ct = ch.CellType_GetPointer()[o];
      if (ct.GetIsNoDelete()) f |= MAC_FLAG_NODELETE;
      out.flags[idx] = f;
      out.type[idx] = (uint8_t)m_celltype2.MaterialToInt(ct.m_mat);
      out.layer[idx] = ch.Layer_GetPointer()[o].GetLayer();
      out.id[idx] = ch.Id_Cell_GetPointer()[o].GetLayer();
#ifdef MAC_DEPTH
      out.depth[idx] = ch.Depth_GetPointer()[o].GetDepth();
#else
      out.depth[idx] = -1;
#endif
    }
    ++c;
  }
  int64_t q = 0;
  for (auto it = plist.begin(); it != plist.end(); ++it, ++q) {
    const auto& v = (*it).GetParticlePos();
    out.pos[3 * q] = v.Get(1); out.pos[3 * q + 1] = v.Get(2); out.pos[3 * q + 2] = v.Get(3);
  }
  if (mac_state_write(argv[3], &out) != 0) { fprintf(stderr, "cannot write %s\n", argv[3]); return 1; }
  mac_state_free(&out);
  mac_state_free(&st);
  SingletonManager::Kill();
  return 0;
}

int main(int argc, char** argv) { return run(argc, argv); }
