// tlm_kernels.cuh -- sm_100a kernels of the SCN-TLM time step.
//
// One time step of GGI_TLM (SRC/TLM_SOLVER/run_TLM.F90:240-293) is
//   excitation -> scatter -> cell_output -> connect -> face_output -> outer_boundary.
// Here it is re-formulated as a "pull" step over structure-of-arrays
// reflected-pulse planes held in a ping-pong pair of buffers:
//
//   tlm_cell_kernel   : for every cell, gather the 12 incident pulses from the
//                       neighbours' reflected pulses of the previous step (this
//                       *is* the free-space connect, connect_normal_to_*.F90:1-10,
//                       and the outer-boundary reflection, outer_boundary.F90:71-131,
//                       read through ghost slots), scatter (scatter.F90,
//                       scatter_PML.F90) and write the 12 reflected pulses.
//                       12 plane reads + 12 plane writes per cell: one HBM pass.
//   tlm_face_kernel   : the few special faces (Huygens excitation faces, output
//                       faces) re-do their connect with the reference's formulas
//                       (connect_normal_to_*.F90:287-360) in place on the
//                       reflected planes and record face fields.
//   tlm_dft_kernel    : FP64 frequency-domain accumulation on output faces
//                       (frequency_output_surfaces.F90:405-406).
//
// Plane layout: element (x,y,z) of every port plane lives at
//   ((z+1)*Py + (y+1))*Px + x,   Px = roundup(nx+1, 4), Py = ny+2, Pz = nz+2,
// so x=-1 / x=nx, y=-1 / y=ny and z=-1 / z=nz are ghost slots.  A ghost slot
// holds R * (the boundary cell's own reflected pulse), written by that cell,
// which is exactly what the reference's outer_boundary leaves in the boundary
// port before the next scatter.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace tlm {

// SRC/CONSTANTS/constants.F90:27-39
constexpr double kZ0 = 376.73031346177;
constexpr double kY0 = 1.0 / 376.73031346177;

// port numbering, SRC/TLM_MODULES/Mesh_Modules.F90:83-94 (0-based)
enum Port {
  Vy_xmin = 0, Vz_xmin, Vy_xmax, Vz_xmax, Vx_ymin, Vz_ymin,
  Vx_ymax, Vz_ymax, Vx_zmin, Vy_zmin, Vx_zmax, Vy_zmax
};
// PML paper notation, SRC/TLM_MODULES/PML_module.F90:59-70
enum PmlPort {
  Vxny = 0, Vxnz, Vxpy, Vxpz, Vynx, Vynz, Vypx, Vypz, Vznx, Vzny, Vzpx, Vzpy
};

enum SpecialFlags : int { SP_MAT = 2, SP_EXC = 4, SP_OUT = 8 };

constexpr int kMaxOrder = 8;
// PML state: 18 values per cell.  scatter_PML.F90 keeps 24 (last I x3, the
// 12 incident pulses, Vxt/Vyt/Vzt, six series voltages), but its STAGE 5
// reads the 12 pulses only as six sums of opposite-port pairs, so the
// pairs are stored instead: slots 0-2 last I, 3-8 the pair sums
// (znx+zpx, ynx+ypx | xny+xpy, zny+zpy | ynz+ypz, xnz+xpz), 9-11 Vt, 12-17
// the series voltages.  Layout: tiles of 32 cells, each holding the values
// as runs of 32 words ([n/32][18][32]), so a warp's state is one contiguous
// 2.25 KB (FP32) or 4.5 KB (FP64) block instead of 18 separate streams.
constexpr int kPmlState = 18;
__host__ __device__ __forceinline__ size_t pml_sidx(int k, long long s) {
  return ((size_t)(s >> 5) * kPmlState + (size_t)k) * 32 + (size_t)(s & 31);
}
__host__ __device__ __forceinline__ size_t pml_state_elems(long long n) {
  return (size_t)((n + 31) / 32) * kPmlState * 32;
}

// FP32 path: free-space scatter arithmetic in FP64 on the FP32 links.  A
// static field (the charge a Gaussian point source leaves) repeats the same
// FP32 rounding every step, and the probes drift; with one rounding per
// stored pulse the 512^3 point-source mesh goes from 1.25e-4 to 2.5e-5
// relative L2 against FP64 over 2000 steps, for ~1% of step time.
#ifndef TLM_FP32_SCATTER_FP64
#define TLM_FP32_SCATTER_FP64 1
#endif

// PML-list parameter index of a PML cell inside a volume material (those
// cells take tlm_pml_material_kernel)
constexpr uint16_t kPmlMaterialSlot = 0xFFFF;
// Bit 15 of a PML cell's parameter index marks an output cell (rows < 2^15).
constexpr int kPmlOutputFlag = 0x8000;

// One volume material after calculate_volume_material_filter_coefficients.
struct MatDev {
  int type, eps_exists, mu_exists, eps_order, mu_order, pad0, pad1, pad2;
  double Ys_eps_f, Zs_mu_f, Ge, Rm;
  // reciprocals of the material's constant divisors (the Thevenin sums and
  // the filters' b(0)), so the per-cell update multiplies instead of running
  // IEEE FP64 divisions; the reference's build (-funsafe-math-optimizations)
  // licenses the same rewrite
  double inv_eps_b0, inv_mu_b0, inv_Y_eps, inv_Y_Ge, inv_Z;
  double eps_a[kMaxOrder + 1], eps_b[kMaxOrder + 1], mu_a[kMaxOrder + 1], mu_b[kMaxOrder + 1];
};

// Storage and arithmetic types of the PML update for a link type T.
template <typename T> struct PmlTypes { using state = T; using arith = T; };
template <> struct PmlTypes<float> {
  using state = float;
  // The PML recursions run in FP64 with FP64 coefficients: with FP32
  // coefficients (exp(-s dt/2), 1-(s_i+s_j)dt/4, ...) the quasi-static field a
  // DC-carrying source leaves inside the PML drifts, and the late-time probe
  // error grows 100x.  The state stays FP32 in storage.
  using arith = double;
};

template <typename T>
struct MeshDev {
  int nx, ny, nz, Px, Py;
  long long PxPy;           // elements per z-plane (incl. ghost rows)
  long long plane;          // elements per port plane
  int chunks_per_plane;     // ny*Px/VEC
  int segs_per_plane;       // ceil(ny*Px/32)
  T *links0, *links1;       // 12 planes each
  T R[6];
  const uint32_t *seg_mask;
  const uint32_t *seg_base;
  const int4 *sp_rec;
  const int4 *sp_pos;       // (x, y, z) 0-based of each special cell
  typename PmlTypes<T>::state *pml_state;  // [n_pml/32][18][32], pml_sidx
  int n_pml;
  const double *pml_par;    // [n_par][16], FP64 in both precisions
  typename PmlTypes<T>::state *pml_ixt;    // [n_out][3]
  double *filt;             // [J][n_filt]
  int n_filt, filt_eo, filt_mo;  // eps/mu max orders (state taps per component)
  const MatDev *mats;
  const double *exc_field;  // [n_timesteps][n_exc][9]
  const int8_t *exc_type;   // [n_exc][6]
  int n_exc;
  double *cell_out;         // [n_timesteps][n_hist][6]: outputs that keep a time series
  double *cell_cur;         // [n_out][6]: every output cell's fields at the current step
  const int *out_hist;      // [n_out]: slot in cell_out, or -1 (no time series)
  int n_out, n_hist;
  double dl, dt;
  const int *d_base;        // device step counter (1-based step of relative step 0)
  int wrap;                 // wrapping boundaries: bit 0 x, bit 1 y, bit 2 z (wrap_outer_boundary.F90)
  // bytes added to what every bulk-copy wait of the TMA cell kernel expects:
  // 0, except under tlm_gpu_set_test_wait_pad (the waits then run out)
  uint32_t tx_pad;
};

// The ghost slot a boundary cell writes: R times its reflected pulse on a
// boundary port, where the neighbour across that boundary pulls it next
// step.  Without wrapping that is the cell itself (outer_boundary.F90:
// 71-131: the port keeps R times its pulse); with wrapping on that axis it is
// the cell at the opposite end of the same row (wrap_outer_boundary.F90:
// 101-273 swaps the two ends' ports after outer_boundary).  port: the
// reflected port on the boundary; opp: the port on the same axis at the
// other end; back: the element shift from the cell to its own ghost slot
// (-1, +1, -dy, +dy, -dz, +dz); span: the shift to the ghost slot past the
// other end (n elements along the axis, with back's sign flipped).
template <typename T>
__device__ __forceinline__ void ghost(T *out, long long P, long long idx, bool wrap, int port, int opp,
                                      long long back, long long span, T v) {
  if (wrap) out[port * P + idx + span] = v;
  else out[opp * P + idx + back] = v;
}

// All ghost writes of one boundary cell at (x, y, z) with reflected pulses co.
template <typename T>
__device__ __forceinline__ void write_ghosts(const MeshDev<T> &m, T *out, long long idx, int x, int y, int z,
                                             const T (&co)[12]) {
  const long long P = m.plane, dy = m.Px, dz = m.PxPy;
  const bool wx = m.wrap & 1, wy = m.wrap & 2, wz = m.wrap & 4;
  if (x == 0) {
    ghost(out, P, idx, wx, Vy_xmin, Vy_xmax, -1, (long long)m.nx, m.R[0] * co[Vy_xmin]);
    ghost(out, P, idx, wx, Vz_xmin, Vz_xmax, -1, (long long)m.nx, m.R[0] * co[Vz_xmin]);
  }
  if (x == m.nx - 1) {
    ghost(out, P, idx, wx, Vy_xmax, Vy_xmin, 1, -(long long)m.nx, m.R[1] * co[Vy_xmax]);
    ghost(out, P, idx, wx, Vz_xmax, Vz_xmin, 1, -(long long)m.nx, m.R[1] * co[Vz_xmax]);
  }
  if (y == 0) {
    ghost(out, P, idx, wy, Vx_ymin, Vx_ymax, -dy, m.ny * dy, m.R[2] * co[Vx_ymin]);
    ghost(out, P, idx, wy, Vz_ymin, Vz_ymax, -dy, m.ny * dy, m.R[2] * co[Vz_ymin]);
  }
  if (y == m.ny - 1) {
    ghost(out, P, idx, wy, Vx_ymax, Vx_ymin, dy, -m.ny * dy, m.R[3] * co[Vx_ymax]);
    ghost(out, P, idx, wy, Vz_ymax, Vz_ymin, dy, -m.ny * dy, m.R[3] * co[Vz_ymax]);
  }
  if (z == 0) {
    ghost(out, P, idx, wz, Vx_zmin, Vx_zmax, -dz, m.nz * dz, m.R[4] * co[Vx_zmin]);
    ghost(out, P, idx, wz, Vy_zmin, Vy_zmax, -dz, m.nz * dz, m.R[4] * co[Vy_zmin]);
  }
  if (z == m.nz - 1) {
    ghost(out, P, idx, wz, Vx_zmax, Vx_zmin, dz, -m.nz * dz, m.R[5] * co[Vx_zmax]);
    ghost(out, P, idx, wz, Vy_zmax, Vy_zmin, dz, -m.nz * dz, m.R[5] * co[Vy_zmax]);
  }
}

// cell_output_field(out_no, 1:6) of step t (output_points.F90:463-612):
// every output cell writes its current-step row, which the volume outputs
// read; an output that keeps a time series (a probe) also writes row t of
// its series.
template <typename T>
__device__ __forceinline__ void store_cell_out(const MeshDev<T> &m, int t, int out_no, const double (&f)[6]) {
  double *cur = m.cell_cur + (size_t)out_no * 6;
#pragma unroll
  for (int c = 0; c < 6; c++) cur[c] = f[c];
  const int h = m.out_hist[out_no];
  if (h >= 0) {
    double *row = m.cell_out + ((size_t)(t - 1) * m.n_hist + h) * 6;
#pragma unroll
    for (int c = 0; c < 6; c++) row[c] = f[c];
  }
}

template <typename T, int VEC> struct VecT;
template <> struct VecT<float, 4> { using type = float4; };
template <> struct VecT<double, 2> { using type = double2; };

template <typename T, int VEC>
__device__ __forceinline__ void load_vec(const T *__restrict__ p, T (&v)[VEC]) {
  using V = typename VecT<T, VEC>::type;
  V q = __ldcs(reinterpret_cast<const V *>(p));
  if constexpr (VEC == 4) { v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w; }
  else { v[0] = q.x; v[1] = q.y; }
}

template <typename T, int VEC>
__device__ __forceinline__ void store_vec(T *__restrict__ p, const T (&v)[VEC]) {
  using V = typename VecT<T, VEC>::type;
  V q;
  if constexpr (VEC == 4) { q.x = v[0]; q.y = v[1]; q.z = v[2]; q.w = v[3]; }
  else { q.x = v[0]; q.y = v[1]; }
  __stcs(reinterpret_cast<V *>(p), q);
}

// ---------------------------------------------------------------------------
// Free-space scatter, scatter.F90:222-272 (pull form: inc -> out)
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void scatter_pulses(const T *inc, T *out, T Vx, T Vy, T Vz, T Ix, T Iy, T Iz) {
  const T Z0 = T(kZ0);
  out[Vx_ymin] = Vx - Z0 * Iz - inc[Vx_ymax];
  out[Vx_ymax] = Vx + Z0 * Iz - inc[Vx_ymin];
  out[Vx_zmin] = Vx + Z0 * Iy - inc[Vx_zmax];
  out[Vx_zmax] = Vx - Z0 * Iy - inc[Vx_zmin];
  out[Vy_zmin] = Vy - Z0 * Ix - inc[Vy_zmax];
  out[Vy_zmax] = Vy + Z0 * Ix - inc[Vy_zmin];
  out[Vy_xmin] = Vy + Z0 * Iz - inc[Vy_xmax];
  out[Vy_xmax] = Vy - Z0 * Iz - inc[Vy_xmin];
  out[Vz_xmin] = Vz - Z0 * Iy - inc[Vz_xmax];
  out[Vz_xmax] = Vz + Z0 * Iy - inc[Vz_xmin];
  out[Vz_ymin] = Vz + Z0 * Ix - inc[Vz_ymax];
  out[Vz_ymax] = Vz - Z0 * Ix - inc[Vz_ymin];
}

// In FP64 the formulas follow scatter.F90 literally (I = (...)/(2 Z0), then
// Z0*I).  In FP32 the currents are carried scaled by Z0 (U = Z0*I = (...)/2):
// algebraically identical, one rounding less per current, and halving is
// exact in both precisions.
template <typename T>
__device__ __forceinline__ void free_space_cell(const T *inc, T *out) {
  const T Vx = (inc[Vx_ymin] + inc[Vx_ymax] + inc[Vx_zmin] + inc[Vx_zmax]) / T(2);
  const T Vy = (inc[Vy_xmin] + inc[Vy_xmax] + inc[Vy_zmin] + inc[Vy_zmax]) / T(2);
  const T Vz = (inc[Vz_xmin] + inc[Vz_xmax] + inc[Vz_ymin] + inc[Vz_ymax]) / T(2);
  if constexpr (sizeof(T) == 8) {
    const double Ix = (inc[Vz_ymax] - inc[Vy_zmax] - inc[Vz_ymin] + inc[Vy_zmin]) / (2.0 * kZ0);
    const double Iy = (inc[Vx_zmax] - inc[Vz_xmax] - inc[Vx_zmin] + inc[Vz_xmin]) / (2.0 * kZ0);
    const double Iz = (inc[Vy_xmax] - inc[Vx_ymax] - inc[Vy_xmin] + inc[Vx_ymin]) / (2.0 * kZ0);
    scatter_pulses<T>(inc, out, Vx, Vy, Vz, Ix, Iy, Iz);
  } else if (TLM_FP32_SCATTER_FP64) {
    // FP32 links, FP64 arithmetic: each stored pulse is the once-rounded
    // exact result (static fields otherwise drift by repeating the same
    // FP32 rounding every step)
    double d[12];
#pragma unroll
    for (int k = 0; k < 12; k++) d[k] = double(inc[k]);
    const double vx = (d[Vx_ymin] + d[Vx_ymax] + d[Vx_zmin] + d[Vx_zmax]) * 0.5;
    const double vy = (d[Vy_xmin] + d[Vy_xmax] + d[Vy_zmin] + d[Vy_zmax]) * 0.5;
    const double vz = (d[Vz_xmin] + d[Vz_xmax] + d[Vz_ymin] + d[Vz_ymax]) * 0.5;
    const double ux = (d[Vz_ymax] - d[Vy_zmax] - d[Vz_ymin] + d[Vy_zmin]) * 0.5;
    const double uy = (d[Vx_zmax] - d[Vz_xmax] - d[Vx_zmin] + d[Vz_xmin]) * 0.5;
    const double uz = (d[Vy_xmax] - d[Vx_ymax] - d[Vy_xmin] + d[Vx_ymin]) * 0.5;
    out[Vx_ymin] = T(vx - uz - d[Vx_ymax]);
    out[Vx_ymax] = T(vx + uz - d[Vx_ymin]);
    out[Vx_zmin] = T(vx + uy - d[Vx_zmax]);
    out[Vx_zmax] = T(vx - uy - d[Vx_zmin]);
    out[Vy_zmin] = T(vy - ux - d[Vy_zmax]);
    out[Vy_zmax] = T(vy + ux - d[Vy_zmin]);
    out[Vy_xmin] = T(vy + uz - d[Vy_xmax]);
    out[Vy_xmax] = T(vy - uz - d[Vy_xmin]);
    out[Vz_xmin] = T(vz - uy - d[Vz_xmax]);
    out[Vz_xmax] = T(vz + uy - d[Vz_xmin]);
    out[Vz_ymin] = T(vz + ux - d[Vz_ymax]);
    out[Vz_ymax] = T(vz - ux - d[Vz_ymin]);
  } else {
    const T Ux = (inc[Vz_ymax] - inc[Vy_zmax] - inc[Vz_ymin] + inc[Vy_zmin]) / T(2);
    const T Uy = (inc[Vx_zmax] - inc[Vz_xmax] - inc[Vx_zmin] + inc[Vz_xmin]) / T(2);
    const T Uz = (inc[Vy_xmax] - inc[Vx_ymax] - inc[Vy_xmin] + inc[Vx_ymin]) / T(2);
    out[Vx_ymin] = Vx - Uz - inc[Vx_ymax];
    out[Vx_ymax] = Vx + Uz - inc[Vx_ymin];
    out[Vx_zmin] = Vx + Uy - inc[Vx_zmax];
    out[Vx_zmax] = Vx - Uy - inc[Vx_zmin];
    out[Vy_zmin] = Vy - Ux - inc[Vy_zmax];
    out[Vy_zmax] = Vy + Ux - inc[Vy_zmin];
    out[Vy_xmin] = Vy + Uz - inc[Vy_xmax];
    out[Vy_xmax] = Vy - Uz - inc[Vy_xmin];
    out[Vz_xmin] = Vz - Uy - inc[Vz_xmax];
    out[Vz_xmax] = Vz + Uy - inc[Vz_xmin];
    out[Vz_ymin] = Vz + Ux - inc[Vz_ymax];
    out[Vz_ymax] = Vz - Ux - inc[Vz_ymin];
  }
}

// ---------------------------------------------------------------------------
// PML free-space cell, scatter_PML.F90:22-313
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void pml_cell(const MeshDev<T> &m, int pidx, const double (&P)[15], int out_no,
                                      const T *inc_in, T *out, int t,
                                      const typename PmlTypes<T>::state (&st)[kPmlState]) {
  using A = typename PmlTypes<T>::arith;
  using ST = typename PmlTypes<T>::state;
  // FP64: literal scatter_PML.F90 arithmetic.  FP32: currents (and the
  // series-term state) carried scaled by Z0, i.e. Z0 = 1 below.
  const A Z0 = sizeof(T) == 8 ? A(kZ0) : A(1);
  // P: the cell's PML_parameters row (TLM_PML_volume_materials.F90:325-351)
  const A ax = A(P[0]), ay = A(P[1]), az = A(P[2]);
  const A exp_x = A(P[3]), exp_y = A(P[4]), exp_z = A(P[5]);
  const A Csx = A(P[6]), Csy = A(P[7]), Csz = A(P[8]);
  const A Csx2 = A(P[9]), Csy2 = A(P[10]), Csz2 = A(P[11]);
  const A Csy_sz = A(P[12]), Csz_sx = A(P[13]), Csx_sy = A(P[14]);
  ST *S = m.pml_state;
  // st: the cell's state as the caller loaded it (slot order of pml_sidx)
  auto ld = [&](int k) -> A { return A(st[k]); };
  const A last_Ix = ld(0), last_Iy = ld(1), last_Iz = ld(2);
  // last incident pulses, as the opposite-port pair sums STAGE 5 uses
  A last_P[6];
#pragma unroll
  for (int k = 0; k < 6; k++) last_P[k] = ld(3 + k);
  const A last_Vxt = ld(9), last_Vyt = ld(10), last_Vzt = ld(11);
  const A last_Vxyt = ld(12), last_Vyxt = ld(13);
  const A last_Vzxt = ld(14), last_Vxzt = ld(15);
  const A last_Vyzt = ld(16), last_Vzyt = ld(17);

  // STAGE 3: half-cell loss on incident pulses
  A V[12];
  V[Vynx] = inc_in[Vynx] * exp_y; V[Vypx] = inc_in[Vypx] * exp_y;
  V[Vznx] = inc_in[Vznx] * exp_z; V[Vzpx] = inc_in[Vzpx] * exp_z;
  V[Vxny] = inc_in[Vxny] * exp_x; V[Vxpy] = inc_in[Vxpy] * exp_x;
  V[Vzny] = inc_in[Vzny] * exp_z; V[Vzpy] = inc_in[Vzpy] * exp_z;
  V[Vxnz] = inc_in[Vxnz] * exp_x; V[Vxpz] = inc_in[Vxpz] * exp_x;
  V[Vynz] = inc_in[Vynz] * exp_y; V[Vypz] = inc_in[Vypz] * exp_y;
  // STAGE 4
  const A Vx = (V[Vynx] + V[Vypx] + V[Vznx] + V[Vzpx]) / A(2);
  const A Vy = (V[Vxny] + V[Vxpy] + V[Vzny] + V[Vzpy]) / A(2);
  const A Vz = (V[Vxnz] + V[Vxpz] + V[Vynz] + V[Vypz]) / A(2);
  // 1/(2 Z0) is a compile-time constant: a multiply, not an FP64 division
  const A inv2Z0 = A(1) / (A(2) * Z0);
  const A Ix = (V[Vypz] - V[Vzpy] - V[Vynz] + V[Vzny]) * inv2Z0;
  const A Iy = (V[Vzpx] - V[Vxpz] - V[Vznx] + V[Vxnz]) * inv2Z0;
  const A Iz = (V[Vxpy] - V[Vypx] - V[Vxny] + V[Vynx]) * inv2Z0;
  // STAGE 5
  A Pn[6];
  Pn[0] = V[Vznx] + V[Vzpx]; Pn[1] = V[Vynx] + V[Vypx];
  Pn[2] = V[Vxny] + V[Vxpy]; Pn[3] = V[Vzny] + V[Vzpy];
  Pn[4] = V[Vynz] + V[Vypz]; Pn[5] = V[Vxnz] + V[Vxpz];
  // The recursions that end in the reported fields (Vxt.., Ixt..) fuse
  // their multiply-adds explicitly, in the reference's association order,
  // so the rounding does not depend on the compiler's choices (and the
  // FP32 kernel fits 96 registers without a spill).
  static_assert(sizeof(A) == 8, "the PML recursion runs in FP64");
  const A Vx_sh = __dmul_rn(ax, __fma_rn(Csy_sz, last_Vxt, __fma_rn(Csz, Pn[1] + last_P[1],
                                         __fma_rn(Csy, Pn[0] + last_P[0], -(last_P[0] + last_P[1]) / A(2)))));
  const A Vy_sh = __dmul_rn(ay, __fma_rn(Csz_sx, last_Vyt, __fma_rn(Csx, Pn[3] + last_P[3],
                                         __fma_rn(Csz, Pn[2] + last_P[2], -(last_P[2] + last_P[3]) / A(2)))));
  const A Vz_sh = __dmul_rn(az, __fma_rn(Csx_sy, last_Vzt, __fma_rn(Csy, Pn[5] + last_P[5],
                                         __fma_rn(Csx, Pn[4] + last_P[4], -(last_P[4] + last_P[5]) / A(2)))));
  // STAGE 6
  const A Vxt = __fma_rn(ax, Vx, Vx_sh), Vyt = __fma_rn(ay, Vy, Vy_sh), Vzt = __fma_rn(az, Vz, Vz_sh);
  // STAGE 7a (output cells only)
  A Ixt = A(0), Iyt = A(0), Izt = A(0);
  if (out_no >= 0) {
    ST *X = m.pml_ixt + (size_t)out_no * 3;
    Ixt = __dmul_rn(ax, __fma_rn(Csy_sz, A(X[0]), __fma_rn(Csx2, Ix + last_Ix, Ix - last_Ix)));
    Iyt = __dmul_rn(ay, __fma_rn(Csz_sx, A(X[1]), __fma_rn(Csy2, Iy + last_Iy, Iy - last_Iy)));
    Izt = __dmul_rn(az, __fma_rn(Csx_sy, A(X[2]), __fma_rn(Csz2, Iz + last_Iz, Iz - last_Iz)));
    X[0] = ST(Ixt); X[1] = ST(Iyt); X[2] = ST(Izt);
  }
  // STAGE 7
  const A Vxy_se = az * (Z0 * (-last_Iz + Csy2 * (Iz + last_Iz)) + Csx_sy * last_Vxyt);
  const A Vyx_se = az * (Z0 * (-last_Iz + Csx2 * (Iz + last_Iz)) + Csx_sy * last_Vyxt);
  const A Vzx_se = ay * (Z0 * (-last_Iy + Csx2 * (Iy + last_Iy)) + Csz_sx * last_Vzxt);
  const A Vxz_se = ay * (Z0 * (-last_Iy + Csz2 * (Iy + last_Iy)) + Csz_sx * last_Vxzt);
  const A Vyz_se = ax * (Z0 * (-last_Ix + Csz2 * (Ix + last_Ix)) + Csy_sz * last_Vyzt);
  const A Vzy_se = ax * (Z0 * (-last_Ix + Csy2 * (Ix + last_Ix)) + Csy_sz * last_Vzyt);
  // STAGE 8 + 9: save state
  __stcs(S + pml_sidx(0, pidx), ST(Ix)); __stcs(S + pml_sidx(1, pidx), ST(Iy)); __stcs(S + pml_sidx(2, pidx), ST(Iz));
#pragma unroll
  for (int k = 0; k < 6; k++) __stcs(S + pml_sidx(3 + k, pidx), ST(Pn[k]));
  __stcs(S + pml_sidx(9, pidx), ST(Vxt)); __stcs(S + pml_sidx(10, pidx), ST(Vyt)); __stcs(S + pml_sidx(11, pidx), ST(Vzt));
  __stcs(S + pml_sidx(12, pidx), ST(az * Iz * Z0 + Vxy_se));
  __stcs(S + pml_sidx(13, pidx), ST(az * Iz * Z0 + Vyx_se));
  __stcs(S + pml_sidx(14, pidx), ST(ay * Iy * Z0 + Vzx_se));
  __stcs(S + pml_sidx(15, pidx), ST(ay * Iy * Z0 + Vxz_se));
  __stcs(S + pml_sidx(16, pidx), ST(ax * Ix * Z0 + Vyz_se));
  __stcs(S + pml_sidx(17, pidx), ST(ax * Ix * Z0 + Vzy_se));
  // STAGE 10
  const A Vynx_P = Vx_sh - Vyx_se, Vypx_P = Vx_sh + Vyx_se;
  const A Vznx_P = Vx_sh + Vzx_se, Vzpx_P = Vx_sh - Vzx_se;
  const A Vxny_P = Vy_sh + Vxy_se, Vxpy_P = Vy_sh - Vxy_se;
  const A Vzny_P = Vy_sh - Vzy_se, Vzpy_P = Vy_sh + Vzy_se;
  const A Vynz_P = Vz_sh + Vyz_se, Vypz_P = Vz_sh - Vyz_se;
  const A Vxnz_P = Vz_sh - Vxz_se, Vxpz_P = Vz_sh + Vxz_se;
  // STAGE 11 + 13: scattered pulses with half-cell loss
  out[Vynx] = T((ax * Vx - az * Z0 * Iz - V[Vypx] + Vynx_P) * exp_y);
  out[Vypx] = T((ax * Vx + az * Z0 * Iz - V[Vynx] + Vypx_P) * exp_y);
  out[Vznx] = T((ax * Vx + ay * Z0 * Iy - V[Vzpx] + Vznx_P) * exp_z);
  out[Vzpx] = T((ax * Vx - ay * Z0 * Iy - V[Vznx] + Vzpx_P) * exp_z);
  out[Vzny] = T((ay * Vy - ax * Z0 * Ix - V[Vzpy] + Vzny_P) * exp_z);
  out[Vzpy] = T((ay * Vy + ax * Z0 * Ix - V[Vzny] + Vzpy_P) * exp_z);
  out[Vxny] = T((ay * Vy + az * Z0 * Iz - V[Vxpy] + Vxny_P) * exp_x);
  out[Vxpy] = T((ay * Vy - az * Z0 * Iz - V[Vxny] + Vxpy_P) * exp_x);
  out[Vxnz] = T((az * Vz - ay * Z0 * Iy - V[Vxpz] + Vxnz_P) * exp_x);
  out[Vxpz] = T((az * Vz + ay * Z0 * Iy - V[Vxnz] + Vxpz_P) * exp_x);
  out[Vynz] = T((az * Vz + ax * Z0 * Ix - V[Vypz] + Vynz_P) * exp_y);
  out[Vypz] = T((az * Vz - ax * Z0 * Ix - V[Vynz] + Vypz_P) * exp_y);
  // STAGE 12: output
  if (out_no >= 0) {
    const double dl = m.dl;
    const double hs = sizeof(T) == 8 ? dl : dl * kZ0;  // FP32 carries Z0*I
    const double f[6] = {-double(Vxt) / dl, -double(Vyt) / dl, -double(Vzt) / dl,
                         double(Ixt) / hs,  double(Iyt) / hs,  double(Izt) / hs};
    store_cell_out(m, t, out_no, f);
  }
}

// evaluate_Zfilter (filter_subroutines.F90:510-540) on a state whose taps
// w(1..order) are given; returns f and sets w0.
// MAXO is a compile-time bound on the order: the loops unroll with the
// runtime order as a predicate, so the taps stay in registers.
template <int MAXO>
__device__ __forceinline__ double zfilter_eval(const double *a, const double *b, double inv_b0, int order,
                                               const double *w, double G, double &w0) {
  double W0 = G;
#pragma unroll
  for (int i = 1; i <= MAXO; i++)
    if (i <= order) W0 = W0 - b[i] * w[i];
  W0 = W0 * inv_b0;
  w0 = W0;
  double F0 = 0.0;
  F0 = F0 + a[0] * W0;
#pragma unroll
  for (int i = 1; i <= MAXO; i++)
    if (i <= order) F0 = F0 + a[i] * w[i];
  return F0;
}

// ---------------------------------------------------------------------------
// Material / excitation / output cell (not PML), scatter.F90:274-547, in FP64
// ---------------------------------------------------------------------------
// MAXO: compile-time bound on every material's eps and mu filter order in the mesh.
// s: the record index, which is also the cell's slot in the filter-tap
// arrays (one slot per record), so the taps can be loaded before the
// record and its material are known.
template <typename T, int MAXO>
__device__ __forceinline__ void special_cell(const MeshDev<T> &m, int s, int4 rec, int t, const T *incT, T *outT) {
  const int flags = rec.x & 0xff;
  const int material = rec.x >> 8;
  double inc[12];
#pragma unroll
  for (int k = 0; k < 12; k++) inc[k] = double(incT[k]);
  const double Z04 = kZ0 * 4.0, Y04 = kY0 * 4.0;
  double VEx = (inc[Vx_ymin] + inc[Vx_ymax] + inc[Vx_zmin] + inc[Vx_zmax]) / 2.0;
  double VEy = (inc[Vy_xmin] + inc[Vy_xmax] + inc[Vy_zmin] + inc[Vy_zmax]) / 2.0;
  double VEz = (inc[Vz_xmin] + inc[Vz_xmax] + inc[Vz_ymin] + inc[Vz_ymax]) / 2.0;
  double Yx = Y04, Yy = Y04, Yz = Y04;
  double VHx = 2.0 * (inc[Vz_ymax] - inc[Vy_zmax] - inc[Vz_ymin] + inc[Vy_zmin]);
  double VHy = 2.0 * (inc[Vx_zmax] - inc[Vz_xmax] - inc[Vx_zmin] + inc[Vz_xmin]);
  double VHz = 2.0 * (inc[Vy_xmax] - inc[Vx_ymax] - inc[Vy_xmin] + inc[Vx_ymin]);
  double Zx = Z04, Zy = Z04, Zz = Z04;
  double Vo[3] = {0, 0, 0}, Ys = 0.0;
  double we[3][MAXO + 1], wm[3][MAXO + 1];
  const MatDev *M = nullptr;
  int type = 0;
  const int fidx = s;
  // taps w(1..order) of every filter up to the mesh's largest orders
  // (timeshift_Zfilter: w(i) <- w(i-1)); slots past a material's own order
  // are loaded but not used
#pragma unroll
  for (int c = 0; c < 3; c++) {
#pragma unroll
    for (int k = 0; k < MAXO; k++) {
      if (k < m.filt_eo) we[c][k + 1] = m.filt[(size_t)(c * m.filt_eo + k) * m.n_filt + fidx];
      if (k < m.filt_mo) wm[c][k + 1] = m.filt[(size_t)(3 * m.filt_eo + c * m.filt_mo + k) * m.n_filt + fidx];
    }
  }
  if (flags & SP_MAT) {
    M = m.mats + (material - 1);
    type = M->type;
  }
  if (type == 1) {
    VEx = 0.0; VEy = 0.0; VEz = 0.0;
  } else if (type == 2) {
    VHx = 0.0; VHy = 0.0; VHz = 0.0;
  } else if (type == 3) {
    if (M->eps_exists) {
      Ys = M->Ys_eps_f;
      const int o = M->eps_order;
      for (int c = 0; c < 3; c++) Vo[c] = zfilter_eval<MAXO>(M->eps_a, M->eps_b, M->inv_eps_b0, o, we[c], 0.0, we[c][0]);
      double V1, Y1;
      const double iY = M->inv_Y_eps;  // 1 / (Y04 + Ys)
      V1 = (VEx * Yx + Vo[0] * Ys) * iY; Y1 = Yx + Ys; VEx = V1; Yx = Y1;
      V1 = (VEy * Yy + Vo[1] * Ys) * iY; Y1 = Yy + Ys; VEy = V1; Yy = Y1;
      V1 = (VEz * Yz + Vo[2] * Ys) * iY; Y1 = Yz + Ys; VEz = V1; Yz = Y1;
    }
    const double Ge = M->Ge;
    double V1, Y1;
    const double iG = M->inv_Y_Ge;  // 1 / (Y + Ge)
    V1 = (VEx * Yx + 0.0 * Ge) * iG; Y1 = Yx + Ge; VEx = V1; Yx = Y1;
    V1 = (VEy * Yy + 0.0 * Ge) * iG; Y1 = Yy + Ge; VEy = V1; Yy = Y1;
    V1 = (VEz * Yz + 0.0 * Ge) * iG; Y1 = Yz + Ge; VEz = V1; Yz = Y1;
    if (M->mu_exists) {
      const double Zs = M->Zs_mu_f;
      const int o = M->mu_order;
      double Vs[3];
      for (int c = 0; c < 3; c++) Vs[c] = zfilter_eval<MAXO>(M->mu_a, M->mu_b, M->inv_mu_b0, o, wm[c], 0.0, wm[c][0]);
      VHx = VHx + Vs[0]; Zx = Zx + Zs;
      VHy = VHy + Vs[1]; Zy = Zy + Zs;
      VHz = VHz + Vs[2]; Zz = Zz + Zs;
    }
    const double Rm = M->Rm;
    VHx = VHx + 0.0; Zx = Zx + Rm;
    VHy = VHy + 0.0; Zy = Zy + Rm;
    VHz = VHz + 0.0; Zz = Zz + Rm;
  }
  double Vx = VEx, Vy = VEy, Vz = VEz;
  double Ix, Iy, Iz;
  if (type == 3) {  // Zx = Zy = Zz, a material constant
    const double iZ = M->inv_Z;
    Ix = VHx * iZ; Iy = VHy * iZ; Iz = VHz * iZ;
  } else {
    Ix = VHx / Zx; Iy = VHy / Zy; Iz = VHz / Zz;
  }
  if (flags & SP_EXC) {
    // scatter.F90:429-450
    const int e = rec.z;
    const double *field = m.exc_field + ((size_t)(t - 1) * m.n_exc + e) * 9;
    const int8_t *h = m.exc_type + (size_t)e * 6;
    const double dl = m.dl;
    const double Isx = field[6] * dl * dl, Isy = field[7] * dl * dl, Isz = field[8] * dl * dl;
    Vx = double(h[0]) * Vx - field[0] * dl / 2.0 + Isx / Yx;
    Vy = double(h[1]) * Vy - field[1] * dl / 2.0 + Isy / Yy;
    Vz = double(h[2]) * Vz - field[2] * dl / 2.0 + Isz / Yz;
    Ix = double(h[3]) * Ix + field[3] * dl / 2.0;
    Iy = double(h[4]) * Iy + field[4] * dl / 2.0;
    Iz = double(h[5]) * Iz + field[5] * dl / 2.0;
  }
  if (flags & SP_OUT) {
    // scatter.F90:465-480
    const double dl = m.dl;
    const double f[6] = {-Vx / dl, -Vy / dl, -Vz / dl, Ix / dl, Iy / dl, Iz / dl};
    store_cell_out(m, t, rec.w, f);
  }
  if (type == 3) {
    // filter update, scatter.F90:483-515; store taps w(0..order-1)
    if (M->eps_exists) {
      const int o = M->eps_order;
      const double Io[3] = {(Vx - Vo[0]) * Ys, (Vy - Vo[1]) * Ys, (Vz - Vo[2]) * Ys};
      for (int c = 0; c < 3; c++) {
        zfilter_eval<MAXO>(M->eps_a, M->eps_b, M->inv_eps_b0, o, we[c], Io[c], we[c][0]);
#pragma unroll
        for (int k = 0; k < MAXO; k++)
          if (k < o) m.filt[(size_t)(c * m.filt_eo + k) * m.n_filt + fidx] = we[c][k];
      }
    }
    if (M->mu_exists) {
      const int o = M->mu_order;
      const double G[3] = {-Ix, -Iy, -Iz};
      for (int c = 0; c < 3; c++) {
        zfilter_eval<MAXO>(M->mu_a, M->mu_b, M->inv_mu_b0, o, wm[c], G[c], wm[c][0]);
#pragma unroll
        for (int k = 0; k < MAXO; k++)
          if (k < o) m.filt[(size_t)(3 * m.filt_eo + c * m.filt_mo + k) * m.n_filt + fidx] = wm[c][k];
      }
    }
  }
  // scatter.F90:519-547
  double out[12];
  const double Z0 = kZ0;
  out[Vx_ymin] = Vx - Z0 * Iz - inc[Vx_ymax];
  out[Vx_ymax] = Vx + Z0 * Iz - inc[Vx_ymin];
  out[Vx_zmin] = Vx + Z0 * Iy - inc[Vx_zmax];
  out[Vx_zmax] = Vx - Z0 * Iy - inc[Vx_zmin];
  out[Vy_zmin] = Vy - Z0 * Ix - inc[Vy_zmax];
  out[Vy_zmax] = Vy + Z0 * Ix - inc[Vy_zmin];
  out[Vy_xmin] = Vy + Z0 * Iz - inc[Vy_xmax];
  out[Vy_xmax] = Vy - Z0 * Iz - inc[Vy_xmin];
  out[Vz_xmin] = Vz - Z0 * Iy - inc[Vz_xmax];
  out[Vz_xmax] = Vz + Z0 * Iy - inc[Vz_xmin];
  out[Vz_ymin] = Vz + Z0 * Ix - inc[Vz_ymax];
  out[Vz_ymax] = Vz - Z0 * Ix - inc[Vz_ymin];
#pragma unroll
  for (int k = 0; k < 12; k++) outT[k] = T(out[k]);
}

// ---------------------------------------------------------------------------
// Bulk kernel: gather (connect + outer boundary) + free-space scatter for all
// non-special cells.  grid = (ceil(chunks_per_plane/blockDim), nz); one thread
// = VEC consecutive x-cells.  Special cells are skipped (their stores are
// masked out; warps made only of special or out-of-range cells return early)
// and are done by tlm_special_kernel from the same input buffer.
// ---------------------------------------------------------------------------
template <typename T, int VEC>
__global__ void __launch_bounds__(256) tlm_cell_kernel(const MeshDev<T> m, int rel_step) {
  const int z = blockIdx.y;
  const int chunk = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = chunk < m.chunks_per_plane;
  const int lane = threadIdx.x & 31;
  const int e = chunk * VEC;  // element offset in the plane interior
  uint32_t mine = 0;
  int nvalid = 0, y = 0, x0 = 0;
  if (valid) {
    y = e / m.Px;
    x0 = e - y * m.Px;
    nvalid = min(VEC, m.nx - x0);
    const uint32_t mask = __ldg(m.seg_mask + (size_t)z * m.segs_per_plane + (e >> 5));
    mine = (mask >> (e & 31)) & ((1u << VEC) - 1u);
  }
  const uint32_t need = (nvalid > 0) ? (((1u << nvalid) - 1u) & ~mine) : 0u;  // cells to write
  if (__all_sync(0xffffffffu, need == 0)) return;
  const int t = *m.d_base + rel_step;  // 1-based timestep
  const T *__restrict__ in = (t & 1) ? m.links0 : m.links1;   // R_{t-1}
  T *__restrict__ out = (t & 1) ? m.links1 : m.links0;        // R_t
  const long long P = m.plane;
  const long long idx = (long long)(z + 1) * m.PxPy + (long long)m.Px + e;
  const long long dy = m.Px, dz = m.PxPy;

  T inc[12][VEC];
  if (valid) {
    load_vec<T, VEC>(in + Vx_ymax * P + idx - dy, inc[Vx_ymin]);
    load_vec<T, VEC>(in + Vz_ymax * P + idx - dy, inc[Vz_ymin]);
    load_vec<T, VEC>(in + Vx_ymin * P + idx + dy, inc[Vx_ymax]);
    load_vec<T, VEC>(in + Vz_ymin * P + idx + dy, inc[Vz_ymax]);
    load_vec<T, VEC>(in + Vx_zmax * P + idx - dz, inc[Vx_zmin]);
    load_vec<T, VEC>(in + Vy_zmax * P + idx - dz, inc[Vy_zmin]);
    load_vec<T, VEC>(in + Vx_zmin * P + idx + dz, inc[Vx_zmax]);
    load_vec<T, VEC>(in + Vy_zmin * P + idx + dz, inc[Vy_zmax]);
  }
  {
    // x neighbours: own aligned chunk + one element from the neighbouring lane
    T a[VEC], b[VEC], c[VEC], d[VEC];
#pragma unroll
    for (int j = 0; j < VEC; j++) { a[j] = T(0); b[j] = T(0); c[j] = T(0); d[j] = T(0); }
    if (valid) {
      load_vec<T, VEC>(in + Vy_xmax * P + idx, a);
      load_vec<T, VEC>(in + Vz_xmax * P + idx, b);
      load_vec<T, VEC>(in + Vy_xmin * P + idx, c);
      load_vec<T, VEC>(in + Vz_xmin * P + idx, d);
    }
    T pa = __shfl_up_sync(0xffffffffu, a[VEC - 1], 1);
    T pb = __shfl_up_sync(0xffffffffu, b[VEC - 1], 1);
    T nc = __shfl_down_sync(0xffffffffu, c[0], 1);
    T nd = __shfl_down_sync(0xffffffffu, d[0], 1);
    if (valid && lane == 0) {
      pa = in[Vy_xmax * P + idx - 1];
      pb = in[Vz_xmax * P + idx - 1];
    }
    if (valid && lane == 31) {
      nc = in[Vy_xmin * P + idx + VEC];
      nd = in[Vz_xmin * P + idx + VEC];
    }
    inc[Vy_xmin][0] = pa;
    inc[Vz_xmin][0] = pb;
#pragma unroll
    for (int j = 1; j < VEC; j++) { inc[Vy_xmin][j] = a[j - 1]; inc[Vz_xmin][j] = b[j - 1]; }
#pragma unroll
    for (int j = 0; j < VEC - 1; j++) { inc[Vy_xmax][j] = c[j + 1]; inc[Vz_xmax][j] = d[j + 1]; }
    inc[Vy_xmax][VEC - 1] = nc;
    inc[Vz_xmax][VEC - 1] = nd;
  }
  if (need == 0) return;

  // free-space scatter; results overwrite the cell's own incident slots
#pragma unroll
  for (int j = 0; j < VEC; j++) {
    T ci[12], co[12];
#pragma unroll
    for (int p = 0; p < 12; p++) ci[p] = inc[p][j];
    free_space_cell<T>(ci, co);
#pragma unroll
    for (int p = 0; p < 12; p++) inc[p][j] = co[p];
  }
#define res inc

  if (need == (1u << VEC) - 1u) {
#pragma unroll
    for (int p = 0; p < 12; p++) store_vec<T, VEC>(out + p * P + idx, res[p]);
  } else {
#pragma unroll
    for (int j = 0; j < VEC; j++)
      if (need & (1u << j))
#pragma unroll
        for (int p = 0; p < 12; p++) out[p * P + idx + j] = res[p][j];
  }
  // ghost slots: R * own reflected pulse (outer_boundary.F90:71-131)
  if (x0 == 0 && (need & 1u)) {
    ghost(out, P, idx, m.wrap & 1, Vy_xmin, Vy_xmax, -1, (long long)m.nx, m.R[0] * res[Vy_xmin][0]);
    ghost(out, P, idx, m.wrap & 1, Vz_xmin, Vz_xmax, -1, (long long)m.nx, m.R[0] * res[Vz_xmin][0]);
  }
  if (x0 + nvalid == m.nx) {
    const int j = nvalid - 1;  // last cell of the row (selected without dynamic register indexing)
    T vy = res[Vy_xmax][0], vz = res[Vz_xmax][0];
#pragma unroll
    for (int k = 1; k < VEC; k++)
      if (j == k) { vy = res[Vy_xmax][k]; vz = res[Vz_xmax][k]; }
    if (need & (1u << j)) {
      ghost(out, P, idx + j, m.wrap & 1, Vy_xmax, Vy_xmin, 1, -(long long)m.nx, m.R[1] * vy);
      ghost(out, P, idx + j, m.wrap & 1, Vz_xmax, Vz_xmin, 1, -(long long)m.nx, m.R[1] * vz);
    }
  }
  if (y == 0) {
#pragma unroll
    for (int j = 0; j < VEC; j++)
      if (need & (1u << j)) {
        ghost(out, P, idx + j, m.wrap & 2, Vx_ymin, Vx_ymax, -dy, m.ny * dy, m.R[2] * res[Vx_ymin][j]);
        ghost(out, P, idx + j, m.wrap & 2, Vz_ymin, Vz_ymax, -dy, m.ny * dy, m.R[2] * res[Vz_ymin][j]);
      }
  }
  if (y == m.ny - 1) {
#pragma unroll
    for (int j = 0; j < VEC; j++)
      if (need & (1u << j)) {
        ghost(out, P, idx + j, m.wrap & 2, Vx_ymax, Vx_ymin, dy, -m.ny * dy, m.R[3] * res[Vx_ymax][j]);
        ghost(out, P, idx + j, m.wrap & 2, Vz_ymax, Vz_ymin, dy, -m.ny * dy, m.R[3] * res[Vz_ymax][j]);
      }
  }
  if (z == 0) {
#pragma unroll
    for (int j = 0; j < VEC; j++)
      if (need & (1u << j)) {
        ghost(out, P, idx + j, m.wrap & 4, Vx_zmin, Vx_zmax, -dz, m.nz * dz, m.R[4] * res[Vx_zmin][j]);
        ghost(out, P, idx + j, m.wrap & 4, Vy_zmin, Vy_zmax, -dz, m.nz * dz, m.R[4] * res[Vy_zmin][j]);
      }
  }
  if (z == m.nz - 1) {
#pragma unroll
    for (int j = 0; j < VEC; j++)
      if (need & (1u << j)) {
        ghost(out, P, idx + j, m.wrap & 4, Vx_zmax, Vx_zmin, dz, -m.nz * dz, m.R[5] * res[Vx_zmax][j]);
        ghost(out, P, idx + j, m.wrap & 4, Vy_zmax, Vy_zmin, dz, -m.nz * dz, m.R[5] * res[Vy_zmax][j]);
      }
  }
}

#undef res

// ---------------------------------------------------------------------------
// TMA-staged persistent bulk kernel.
//
// Work item = a tile of up to TILE consecutive elements of one z-plane's
// interior (rows y=0..ny-1).  One elected thread per block issues 12
// cp.async.bulk copies (one per source plane segment, shifted by the pull
// offset of that port) into an NSTAGE-deep shared-memory ring completed on an
// mbarrier; the block computes tile i from its stage while the copies of
// tiles i+1.. are in flight.  Results go straight to global memory with
// streaming vector stores.  All mbarrier waits are bounded by %globaltimer;
// on expiry the block records an error code and returns.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// Wait for phase `parity` of an mbarrier, giving up after ~2 s.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (unsigned it = 1;; it++) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 255u) == 0u && global_ns() - t0 > 2000000000ull) return false;
  }
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

constexpr int kErrTimeout = 1;

struct TileList {
  const int4 *tile;  // (z, e0, len, 0)
  int n;
  int *err;          // device error word (0 = ok)
};

template <typename T, int VEC, int TILE, int NSTAGE>
struct TmaCfg {
  static constexpr int H = 16 / (int)sizeof(T);       // halo elements (16 B) on each side of x-planes
  static constexpr int SEG = TILE + 2 * H;             // elements per plane buffer
  static constexpr int THREADS = TILE / VEC;
  static constexpr size_t STAGE_BYTES = (size_t)12 * SEG * sizeof(T);
  static constexpr size_t SMEM = NSTAGE * STAGE_BYTES + 64;
};

template <typename T, int VEC, int TILE, int NSTAGE>
__device__ __forceinline__ void tma_issue(const MeshDev<T> &m, const T *in, const int4 tile, T *stage, uint64_t *bar) {
  using C = TmaCfg<T, VEC, TILE, NSTAGE>;
  const long long P = m.plane;
  const long long idx0 = (long long)(tile.x + 1) * m.PxPy + (long long)m.Px + tile.y;
  const int len = tile.z;
  const uint32_t xb = (uint32_t)((len + 2 * C::H) * sizeof(T));
  const uint32_t yb = (uint32_t)(len * sizeof(T));
  mbar_expect_tx(bar, 4 * xb + 8 * yb + m.tx_pad);
  // buffer b holds the source plane of incident port b (plane of the opposite port)
  const long long dy = m.Px, dz = m.PxPy;
  // x-planes, with a 16-byte halo on both sides
  bulk_g2s(stage + Vy_xmin * C::SEG, in + Vy_xmax * P + idx0 - C::H, xb, bar);
  bulk_g2s(stage + Vz_xmin * C::SEG, in + Vz_xmax * P + idx0 - C::H, xb, bar);
  bulk_g2s(stage + Vy_xmax * C::SEG, in + Vy_xmin * P + idx0 - C::H, xb, bar);
  bulk_g2s(stage + Vz_xmax * C::SEG, in + Vz_xmin * P + idx0 - C::H, xb, bar);
  // y and z planes: the shifted rows/planes, stored at offset H
  bulk_g2s(stage + Vx_ymin * C::SEG + C::H, in + Vx_ymax * P + idx0 - dy, yb, bar);
  bulk_g2s(stage + Vz_ymin * C::SEG + C::H, in + Vz_ymax * P + idx0 - dy, yb, bar);
  bulk_g2s(stage + Vx_ymax * C::SEG + C::H, in + Vx_ymin * P + idx0 + dy, yb, bar);
  bulk_g2s(stage + Vz_ymax * C::SEG + C::H, in + Vz_ymin * P + idx0 + dy, yb, bar);
  bulk_g2s(stage + Vx_zmin * C::SEG + C::H, in + Vx_zmax * P + idx0 - dz, yb, bar);
  bulk_g2s(stage + Vy_zmin * C::SEG + C::H, in + Vy_zmax * P + idx0 - dz, yb, bar);
  bulk_g2s(stage + Vx_zmax * C::SEG + C::H, in + Vx_zmin * P + idx0 + dz, yb, bar);
  bulk_g2s(stage + Vy_zmax * C::SEG + C::H, in + Vy_zmin * P + idx0 + dz, yb, bar);
}

template <typename T, int VEC>
__device__ __forceinline__ void lds_vec(const T *p, T (&v)[VEC]) {
  using V = typename VecT<T, VEC>::type;
  const V q = *reinterpret_cast<const V *>(p);
  if constexpr (VEC == 4) { v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w; }
  else { v[0] = q.x; v[1] = q.y; }
}

// meshes == nullptr: one mesh (m0); otherwise a batch, tile.w indexes meshes[]
template <typename T, int VEC, int TILE, int NSTAGE>
__global__ void __launch_bounds__(TILE / VEC) tlm_bulk_tma_kernel(const MeshDev<T> m0, const MeshDev<T> *meshes,
                                                                  const TileList tl, int rel_step) {
  using C = TmaCfg<T, VEC, TILE, NSTAGE>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T *stages = reinterpret_cast<T *>(smem_raw);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + NSTAGE * C::STAGE_BYTES);
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < NSTAGE; s++) mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const int first = blockIdx.x, stride = gridDim.x;
  int n_mine = (tl.n - first + stride - 1) / stride;
  if (n_mine < 0) n_mine = 0;
  // prologue: fill the ring
  if (tid == 0)
    for (int s = 0; s < NSTAGE && s < n_mine; s++) {
      const int4 tw = tl.tile[first + s * stride];
      const MeshDev<T> &mw = meshes ? meshes[tw.w] : m0;
      const int tt = *mw.d_base + rel_step;
      tma_issue<T, VEC, TILE, NSTAGE>(mw, (tt & 1) ? mw.links0 : mw.links1, tw, stages + s * 12 * C::SEG, &bars[s]);
    }
  for (int i = 0; i < n_mine; i++) {
    const int s = i % NSTAGE;
    const uint32_t parity = (uint32_t)((i / NSTAGE) & 1);
    const int4 tile = tl.tile[first + i * stride];
    const MeshDev<T> &m = meshes ? meshes[tile.w] : m0;
    const int t = *m.d_base + rel_step;
    T *__restrict__ out = (t & 1) ? m.links1 : m.links0;
    const long long P = m.plane;
    const long long dy = m.Px, dz = m.PxPy;
    if (!mbar_wait_bounded(&bars[s], parity)) {
      if (tid == 0) atomicExch(tl.err, kErrTimeout);
      return;
    }
    const T *st = stages + s * 12 * C::SEG;
    const int z = tile.x;
    const int el = tid * VEC;  // element offset inside the tile
    const int e = tile.y + el;
    const bool valid = el < tile.z;
    if (valid) {
      const int y = e / m.Px;
      const int x0 = e - y * m.Px;
      const int nvalid = min(VEC, m.nx - x0);
      const uint32_t mask = __ldg(m.seg_mask + (size_t)z * m.segs_per_plane + (e >> 5));
      const uint32_t mine = (mask >> (e & 31)) & ((1u << VEC) - 1u);
      const uint32_t need = (nvalid > 0) ? (((1u << nvalid) - 1u) & ~mine) : 0u;
      if (need) {
        T inc[12][VEC];
        const int o = C::H + el;
        lds_vec<T, VEC>(st + Vx_ymin * C::SEG + o, inc[Vx_ymin]);
        lds_vec<T, VEC>(st + Vz_ymin * C::SEG + o, inc[Vz_ymin]);
        lds_vec<T, VEC>(st + Vx_ymax * C::SEG + o, inc[Vx_ymax]);
        lds_vec<T, VEC>(st + Vz_ymax * C::SEG + o, inc[Vz_ymax]);
        lds_vec<T, VEC>(st + Vx_zmin * C::SEG + o, inc[Vx_zmin]);
        lds_vec<T, VEC>(st + Vy_zmin * C::SEG + o, inc[Vy_zmin]);
        lds_vec<T, VEC>(st + Vx_zmax * C::SEG + o, inc[Vx_zmax]);
        lds_vec<T, VEC>(st + Vy_zmax * C::SEG + o, inc[Vy_zmax]);
        {
          T a[VEC], b[VEC], c[VEC], d[VEC];
          lds_vec<T, VEC>(st + Vy_xmin * C::SEG + o, a);  // source plane Vy_xmax at x
          lds_vec<T, VEC>(st + Vz_xmin * C::SEG + o, b);
          lds_vec<T, VEC>(st + Vy_xmax * C::SEG + o, c);  // source plane Vy_xmin at x
          lds_vec<T, VEC>(st + Vz_xmax * C::SEG + o, d);
          inc[Vy_xmin][0] = st[Vy_xmin * C::SEG + o - 1];
          inc[Vz_xmin][0] = st[Vz_xmin * C::SEG + o - 1];
#pragma unroll
          for (int j = 1; j < VEC; j++) { inc[Vy_xmin][j] = a[j - 1]; inc[Vz_xmin][j] = b[j - 1]; }
#pragma unroll
          for (int j = 0; j < VEC - 1; j++) { inc[Vy_xmax][j] = c[j + 1]; inc[Vz_xmax][j] = d[j + 1]; }
          inc[Vy_xmax][VEC - 1] = st[Vy_xmax * C::SEG + o + VEC];
          inc[Vz_xmax][VEC - 1] = st[Vz_xmax * C::SEG + o + VEC];
        }
#pragma unroll
        for (int j = 0; j < VEC; j++) {
          T ci[12], co[12];
#pragma unroll
          for (int p = 0; p < 12; p++) ci[p] = inc[p][j];
          free_space_cell<T>(ci, co);
#pragma unroll
          for (int p = 0; p < 12; p++) inc[p][j] = co[p];
        }
        const long long idx = (long long)(z + 1) * m.PxPy + (long long)m.Px + e;
        if (need == (1u << VEC) - 1u) {
#pragma unroll
          for (int p = 0; p < 12; p++) store_vec<T, VEC>(out + p * P + idx, inc[p]);
        } else {
#pragma unroll
          for (int j = 0; j < VEC; j++)
            if (need & (1u << j)) {
#pragma unroll
              for (int p = 0; p < 12; p++) out[p * P + idx + j] = inc[p][j];
            }
        }
        if (x0 == 0 && (need & 1u)) {
          ghost(out, P, idx, m.wrap & 1, Vy_xmin, Vy_xmax, -1, (long long)m.nx, m.R[0] * inc[Vy_xmin][0]);
          ghost(out, P, idx, m.wrap & 1, Vz_xmin, Vz_xmax, -1, (long long)m.nx, m.R[0] * inc[Vz_xmin][0]);
        }
        if (x0 + nvalid == m.nx) {
          const int j = nvalid - 1;
          T vy = inc[Vy_xmax][0], vz = inc[Vz_xmax][0];
#pragma unroll
          for (int k = 1; k < VEC; k++)
            if (j == k) { vy = inc[Vy_xmax][k]; vz = inc[Vz_xmax][k]; }
          if (need & (1u << j)) {
            ghost(out, P, idx + j, m.wrap & 1, Vy_xmax, Vy_xmin, 1, -(long long)m.nx, m.R[1] * vy);
            ghost(out, P, idx + j, m.wrap & 1, Vz_xmax, Vz_xmin, 1, -(long long)m.nx, m.R[1] * vz);
          }
        }
        if (y == 0) {
#pragma unroll
          for (int j = 0; j < VEC; j++)
            if (need & (1u << j)) {
              ghost(out, P, idx + j, m.wrap & 2, Vx_ymin, Vx_ymax, -dy, m.ny * dy, m.R[2] * inc[Vx_ymin][j]);
              ghost(out, P, idx + j, m.wrap & 2, Vz_ymin, Vz_ymax, -dy, m.ny * dy, m.R[2] * inc[Vz_ymin][j]);
            }
        }
        if (y == m.ny - 1) {
#pragma unroll
          for (int j = 0; j < VEC; j++)
            if (need & (1u << j)) {
              ghost(out, P, idx + j, m.wrap & 2, Vx_ymax, Vx_ymin, dy, -m.ny * dy, m.R[3] * inc[Vx_ymax][j]);
              ghost(out, P, idx + j, m.wrap & 2, Vz_ymax, Vz_ymin, dy, -m.ny * dy, m.R[3] * inc[Vz_ymax][j]);
            }
        }
        if (z == 0) {
#pragma unroll
          for (int j = 0; j < VEC; j++)
            if (need & (1u << j)) {
              ghost(out, P, idx + j, m.wrap & 4, Vx_zmin, Vx_zmax, -dz, m.nz * dz, m.R[4] * inc[Vx_zmin][j]);
              ghost(out, P, idx + j, m.wrap & 4, Vy_zmin, Vy_zmax, -dz, m.nz * dz, m.R[4] * inc[Vy_zmin][j]);
            }
        }
        if (z == m.nz - 1) {
#pragma unroll
          for (int j = 0; j < VEC; j++)
            if (need & (1u << j)) {
              ghost(out, P, idx + j, m.wrap & 4, Vx_zmax, Vx_zmin, dz, -m.nz * dz, m.R[5] * inc[Vx_zmax][j]);
              ghost(out, P, idx + j, m.wrap & 4, Vy_zmax, Vy_zmin, dz, -m.nz * dz, m.R[5] * inc[Vy_zmax][j]);
            }
        }
      }
    }
    __syncthreads();  // every thread is done reading stage s
    if (tid == 0 && i + NSTAGE < n_mine) {
      fence_proxy_async();
      const int4 tw = tl.tile[first + (i + NSTAGE) * stride];
      const MeshDev<T> &mw = meshes ? meshes[tw.w] : m0;
      const int tt = *mw.d_base + rel_step;
      tma_issue<T, VEC, TILE, NSTAGE>(mw, (tt & 1) ? mw.links0 : mw.links1, tw, stages + s * 12 * C::SEG, &bars[s]);
    }
  }
}

// ---------------------------------------------------------------------------
// Special-cell kernel: one thread per special cell (traversal order, so PML
// state and links coalesce along x): gather, PML / material / excitation /
// output scatter, reflected pulses + ghost slots.
// ---------------------------------------------------------------------------
template <typename T, int MAXO>
__device__ __forceinline__ void special_body(const MeshDev<T> &m, int s, int rel_step);

template <typename T, int MAXO>
__global__ void __launch_bounds__(128) tlm_special_kernel(const MeshDev<T> m, int n_special, int rel_step) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_special) return;
  special_body<T, MAXO>(m, s, rel_step);
}

template <typename T, int MAXO>
__device__ __forceinline__ void special_body(const MeshDev<T> &m, int s, int rel_step) {
  const int t = *m.d_base + rel_step;
  const T *__restrict__ in = (t & 1) ? m.links0 : m.links1;
  T *__restrict__ out = (t & 1) ? m.links1 : m.links0;
  const long long P = m.plane;
  const int4 pos = m.sp_pos[s];
  const int4 rec = m.sp_rec[s];
  const long long idx = (long long)(pos.z + 1) * m.PxPy + (long long)(pos.y + 1) * m.Px + pos.x;
  const long long dy = m.Px, dz = m.PxPy;
  T ci[12], co[12];
  ci[Vy_xmin] = in[Vy_xmax * P + idx - 1];
  ci[Vz_xmin] = in[Vz_xmax * P + idx - 1];
  ci[Vy_xmax] = in[Vy_xmin * P + idx + 1];
  ci[Vz_xmax] = in[Vz_xmin * P + idx + 1];
  ci[Vx_ymin] = in[Vx_ymax * P + idx - dy];
  ci[Vz_ymin] = in[Vz_ymax * P + idx - dy];
  ci[Vx_ymax] = in[Vx_ymin * P + idx + dy];
  ci[Vz_ymax] = in[Vz_ymin * P + idx + dy];
  ci[Vx_zmin] = in[Vx_zmax * P + idx - dz];
  ci[Vy_zmin] = in[Vy_zmax * P + idx - dz];
  ci[Vx_zmax] = in[Vx_zmin * P + idx + dz];
  ci[Vy_zmax] = in[Vy_zmin * P + idx + dz];
  // PML cells never reach this list: they take tlm_pml_kernel
  special_cell<T, MAXO>(m, s, rec, t, ci, co);
#pragma unroll
  for (int p = 0; p < 12; p++) out[p * P + idx] = co[p];
  write_ghosts<T>(m, out, idx, pos.x, pos.y, pos.z, co);
}

// ---------------------------------------------------------------------------
// PML kernel: one thread per PML cell, in the reference's PML cell numbering
// (traversal order), so the thread index is the PML state index.  Per cell
// it reads an 8-byte packed position (x | y<<21 | z<<42 | output<<63) and a
// 2-byte PML parameter index.
// ---------------------------------------------------------------------------
// Resident 128-thread blocks per SM the PML kernel is compiled for (caps its
// registers at 65536 / (128 x this)).  Measured on B200, 256^3 PML-spheres
// and 512^3 point-source meshes: 3 is 1-5% faster per step than no bound
// (FP64 drops from 184 registers to 170 without spills), 4 and 5 spill and
// are no faster or slower.
#ifndef TLM_PML_MIN_BLOCKS
#define TLM_PML_MIN_BLOCKS 3
#endif
// The FP32 kernel (FP32 state, FP64 arithmetic) fits 4 blocks in 128
// registers without spills, 0.7-1.6 % faster per step than 3; 5 blocks (96
// registers, a 16-byte spill) gains another 0-2 % (C3 and 160^3 most);
// 6 blocks (80 registers, 136-byte spill) is 3-16 % slower.
#ifndef TLM_PML_MIN_BLOCKS_FP32
#define TLM_PML_MIN_BLOCKS_FP32 5
#endif
// L2 prefetch of the link runs a contiguous PML block will gather (with its
// state): 1-3 % per step on PML-bounded meshes.
#ifndef TLM_PML_LINK_PREFETCH
#define TLM_PML_LINK_PREFETCH 1
#endif

// The PML cells of the reference's meshes form a box shell: the cells within
// xl/xh of the x ends, yl/yh of the y ends or zl/zh of the z ends
// (calc_pml_dist).  Numbered in traversal order, a cell's position then
// follows from its PML number, so the link addresses do not wait for a
// position load.
// Division by a constant divisor d >= 1 for dividends 0 <= n < 2^31:
// floor(n / d) = (n * m) >> sh with l = ceil(log2 d), sh = 31 + l and
// m = floor(2^sh / d) + 1 (Granlund and Montgomery, "Division by invariant
// integers using multiplication", PLDI 1994, theorem 4.2: 2^sh < m d <=
// 2^sh + 2^l).  n * m < 2^31 (2^32 + 1) fits 64 bits.
struct FastDiv {
  unsigned long long m;
  int sh;
};
__host__ __device__ __forceinline__ int fast_div(int n, const FastDiv &f) {
  return (int)(((unsigned long long)(unsigned)n * f.m) >> f.sh);
}
inline FastDiv make_fast_div(int d) {
  if (d < 1) d = 1;  // a divisor the decoder never uses
  int l = 0;
  while ((1ll << l) < d) l++;
  FastDiv f;
  f.sh = 31 + l;
  f.m = (1ull << f.sh) / (unsigned long long)d + 1ull;
  return f;
}

struct PmlShell {
  int on;                 // 1: positions from the shell, 0: from `pos`
  int nx, ny, nz, xl, xh, yl, yh, zl, zh;
  int full, partial;      // PML cells of a whole z-plane / of a plane between the z slabs
  FastDiv d_full, d_nx, d_partial, d_w;  // divisors full, nx, partial, xl + xh
};

struct PmlList {
  const unsigned long long *pos;
  const uint16_t *par;
  const int2 *out_map;  // (pml index, output number) of PML output cells, sorted by pml index
  int n, n_out_map;
  PmlShell sh;
  // For a shell whose parameter rows follow the cells' PML distance classes
  // (calc_pml_dist, TLM_PML_volume_materials.F90:446-481; the host checks
  // every cell), the rows indexed by class, [(2 zl+..)][16]: a cell's
  // parameters are then loaded from its position, beside its links and
  // state, instead of after its parameter index arrives.  nullptr: off.
  const double *cls_par;
};

// The PML distance-class index of shell position (x, y, z): per axis the
// signed distance into the PML (-lo..-1 on the low side, 1..hi on the high
// side, 0 outside), offset to 0..lo+hi and combined x fastest.
__host__ __device__ __forceinline__ int pml_class(const PmlShell &h, int x, int y, int z) {
  const int cx = x < h.xl ? x - h.xl : (x >= h.nx - h.xh ? x - (h.nx - h.xh) + 1 : 0);
  const int cy = y < h.yl ? y - h.yl : (y >= h.ny - h.yh ? y - (h.ny - h.yh) + 1 : 0);
  const int cz = z < h.zl ? z - h.zl : (z >= h.nz - h.zh ? z - (h.nz - h.zh) + 1 : 0);
  return ((cz + h.zl) * (h.yl + h.yh + 1) + (cy + h.yl)) * (h.xl + h.xh + 1) + (cx + h.xl);
}

// Position of PML cell s of a shell (traversal order z, y, x).
__host__ __device__ __forceinline__ void pml_shell_pos(const PmlShell &h, int s, int &x, int &y, int &z) {
  const int lo = h.zl * h.full;
  if (s < lo) {
    z = fast_div(s, h.d_full);
    const int r = s - z * h.full;
    y = fast_div(r, h.d_nx);
    x = r - y * h.nx;
    return;
  }
  const int s2 = s - lo;
  const int mid = h.nz - h.zl - h.zh;
  if (s2 < mid * h.partial) {
    const int zz = fast_div(s2, h.d_partial);
    z = h.zl + zz;
    const int r = s2 - zz * h.partial;
    const int rows_lo = h.yl * h.nx;
    if (r < rows_lo) {
      y = fast_div(r, h.d_nx);
      x = r - y * h.nx;
      return;
    }
    const int r2 = r - rows_lo;
    const int w = h.xl + h.xh;
    const int midrows = h.ny - h.yl - h.yh;
    if (r2 < midrows * w) {
      const int yy = fast_div(r2, h.d_w);
      y = h.yl + yy;
      const int c = r2 - yy * w;
      x = c < h.xl ? c : h.nx - h.xh + (c - h.xl);
      return;
    }
    const int r3 = r2 - midrows * w;
    const int yy = fast_div(r3, h.d_nx);
    y = h.ny - h.yh + yy;
    x = r3 - yy * h.nx;
    return;
  }
  const int s3 = s2 - mid * h.partial;
  const int zz = fast_div(s3, h.d_full);
  z = h.nz - h.zh + zz;
  const int r = s3 - zz * h.full;
  y = fast_div(r, h.d_nx);
  x = r - y * h.nx;
}

__device__ __forceinline__ void bulk_prefetch_l2(const void *p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

template <typename T>
__device__ __forceinline__ void pml_body(const MeshDev<T> &m, const PmlList &pl, int s, int rel_step);

// One elected thread pulls into L2 what the PML block of 128 cells starting
// at s0 (a multiple of 128) will read: its state (one contiguous range of
// whole 32-cell tiles), its parameter indices, and its positions or, for a
// shell, the link runs it gathers.  The position range is widened to 16-byte
// boundaries; the position buffer carries 64 bytes of padding so the
// widened range stays inside its allocation.
template <typename T>
__device__ __forceinline__ void pml_prefetch_block(const MeshDev<T> &m, const PmlList &pl, long long s0, int rel_step) {
  const int cnt = (int)min(128LL, (long long)pl.n - s0);
  const long long tiles = ((long long)cnt + 31) / 32;  // s0 is a multiple of 128
  const char *a = reinterpret_cast<const char *>(m.pml_state + pml_sidx(0, s0));
  bulk_prefetch_l2(a, (uint32_t)(tiles * kPmlState * 32 * sizeof(typename PmlTypes<T>::state)));
  // parameter indices: 2 bytes a cell from a 256-byte-aligned start; the
  // index buffer carries 256 bytes of padding
  bulk_prefetch_l2(pl.par + s0, (uint32_t)((cnt * 2 + 15) & ~15));
  if (!pl.sh.on) {
    const char *pa = reinterpret_cast<const char *>(reinterpret_cast<uintptr_t>(pl.pos + s0) & ~(uintptr_t)15);
    bulk_prefetch_l2(pa, (uint32_t)((cnt * 8 + 15) & ~15) + 16);
  } else if (TLM_PML_LINK_PREFETCH) {
    // the links the block will gather, when its cells fill one run of
    // plane elements (z-slab planes, y-slab rows): that run of each
    // source plane, shifted by the port's pull offset and widened to
    // 16-byte boundaries.  idx - 1 >= 0 and idx + dz + 1 < plane for
    // every cell, and planes are whole multiples of 16 bytes, so the
    // widened runs stay inside the link buffer.
    int x0, y0, z0, x1, y1, z1;
    pml_shell_pos(pl.sh, (int)s0, x0, y0, z0);
    pml_shell_pos(pl.sh, (int)(s0 + cnt - 1), x1, y1, z1);
    const long long e0 = (long long)y0 * m.Px + x0, e1 = (long long)y1 * m.Px + x1;
    if (z0 == z1 && e1 - e0 < 2LL * cnt) {
      const int t = *m.d_base + rel_step;
      const T *in = (t & 1) ? m.links0 : m.links1;
      const long long i0 = (long long)(z0 + 1) * m.PxPy + (long long)m.Px + e0;
      const long long len = e1 - e0 + 1;
      const long long P = m.plane, dy = m.Px, dz = m.PxPy;
      const int src[12] = {Vy_xmax, Vz_xmax, Vy_xmin, Vz_xmin, Vx_ymax, Vz_ymax,
                           Vx_ymin, Vz_ymin, Vx_zmax, Vy_zmax, Vx_zmin, Vy_zmin};
      const long long sft[12] = {-1, -1, 1, 1, -dy, -dy, dy, dy, -dz, -dz, dz, dz};
#pragma unroll
      for (int k = 0; k < 12; k++) {
        const uintptr_t b = reinterpret_cast<uintptr_t>(in + src[k] * P + i0 + sft[k]);
        const uintptr_t e = b + (uintptr_t)len * sizeof(T);
        const uintptr_t b16 = b & ~(uintptr_t)15, e16 = (e + 15) & ~(uintptr_t)15;
        bulk_prefetch_l2(reinterpret_cast<const void *>(b16), (uint32_t)(e16 - b16));
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? TLM_PML_MIN_BLOCKS_FP32 : TLM_PML_MIN_BLOCKS) tlm_pml_kernel(const MeshDev<T> m, const PmlList pl, int rel_step,
                                                      int prefetch_blocks) {
  // prefetch for the block that runs prefetch_blocks later, so its loads hit L2
  if (threadIdx.x == 0 && prefetch_blocks > 0) {
    const long long s0 = (long long)(blockIdx.x + prefetch_blocks) * blockDim.x;
    if (s0 < pl.n) pml_prefetch_block<T>(m, pl, s0, rel_step);
  }
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= pl.n) return;
  pml_body<T>(m, pl, s, rel_step);
}

template <typename T>
__device__ __forceinline__ void pml_body(const MeshDev<T> &m, const PmlList &pl, int s, int rel_step) {
  const int t = *m.d_base + rel_step;
  const T *__restrict__ in = (t & 1) ? m.links0 : m.links1;
  T *__restrict__ out = (t & 1) ? m.links1 : m.links0;
  const long long P = m.plane;
  int x, y, z;
  if (pl.sh.on) {
    pml_shell_pos(pl.sh, s, x, y, z);
  } else {
    const unsigned long long pk = __ldcs(pl.pos + s);
    x = (int)(pk & 0x1fffffull); y = (int)((pk >> 21) & 0x1fffffull); z = (int)((pk >> 42) & 0x1fffffull);
  }
  // Every load of the cell is issued before anything waits on one: the
  // parameter index (which also says whether the cell is an output cell or
  // a PML cell in a material) is checked only after the link and state
  // loads are in flight, so a warp waits for one memory round trip, not two.
  const int pw = __ldcs(pl.par + s);
  const long long idx = (long long)(z + 1) * m.PxPy + (long long)(y + 1) * m.Px + x;
  const long long dy = m.Px, dz = m.PxPy;
  T ci[12], co[12];
  ci[Vy_xmin] = __ldcs(in + Vy_xmax * P + idx - 1);
  ci[Vz_xmin] = __ldcs(in + Vz_xmax * P + idx - 1);
  ci[Vy_xmax] = __ldcs(in + Vy_xmin * P + idx + 1);
  ci[Vz_xmax] = __ldcs(in + Vz_xmin * P + idx + 1);
  ci[Vx_ymin] = __ldcs(in + Vx_ymax * P + idx - dy);
  ci[Vz_ymin] = __ldcs(in + Vz_ymax * P + idx - dy);
  ci[Vx_ymax] = __ldcs(in + Vx_ymin * P + idx + dy);
  ci[Vz_ymax] = __ldcs(in + Vz_ymin * P + idx + dy);
  ci[Vx_zmin] = __ldcs(in + Vx_zmax * P + idx - dz);
  ci[Vy_zmin] = __ldcs(in + Vy_zmax * P + idx - dz);
  ci[Vx_zmax] = __ldcs(in + Vx_zmin * P + idx + dz);
  ci[Vy_zmax] = __ldcs(in + Vy_zmin * P + idx + dz);
  // state value k of this cell: S[pml_sidx(k, s)] = S[pml_sidx(0, s) + 32 k]
  using ST = typename PmlTypes<T>::state;
  ST st[kPmlState];
  const ST *Lg = m.pml_state + pml_sidx(0, s);
#pragma unroll
  for (int k = 0; k < kPmlState; k++) st[k] = __ldcs(Lg + 32 * k);
  double prm[15];
  const bool by_class = pl.cls_par != nullptr;
  if (by_class) {  // the parameters from the position: no wait on the index
    const double *row = pl.cls_par + (size_t)pml_class(pl.sh, x, y, z) * 16;
#pragma unroll
    for (int k = 0; k < 15; k++) prm[k] = __ldg(row + k);
  }
  if (pw == kPmlMaterialSlot) return;  // PML cell in a material: tlm_pml_material_kernel
  const int par = pw & (kPmlOutputFlag - 1);
  if (!by_class) {
    const double *row = m.pml_par + (size_t)par * 16;
#pragma unroll
    for (int k = 0; k < 15; k++) prm[k] = row[k];
  }
  int out_no = -1;
  if (pw & kPmlOutputFlag) {  // binary search of the output map (sorted by PML cell)
    int lo = 0, hi = pl.n_out_map - 1;
    while (lo <= hi) {
      const int mid = (lo + hi) >> 1;
      const int2 e = pl.out_map[mid];
      if (e.x == s) { out_no = e.y; break; }
      if (e.x < s) lo = mid + 1; else hi = mid - 1;
    }
  }
  pml_cell<T>(m, s, prm, out_no, ci, co, t, st);
#pragma unroll
  for (int p = 0; p < 12; p++) __stcs(out + p * P + idx, co[p]);
  write_ghosts<T>(m, out, idx, x, y, z, co);
}

// ---------------------------------------------------------------------------
// PML cells inside a non-dispersive volume material,
// TLM_SOLVER/scatter_PML_material.F90:22-534.  One thread per cell; the
// cells keep their slot in the PML numbering (the PML kernel skips them) and
// carry their own FP64 state, 66 values per cell in SoA order:
//   0-11 Vi, 12-23 Vi one step older, 24-26 Vxt..Vzt, 27-29 one step older,
//   30-32 Ixt..Izt, 33-35 one step older, 36-41 series terms (xy yx yz zy zx
//   xz), 42-44 capacitive stub reflected, 45-47 its incident, 48-50 one step
//   older, 51-53 inductive stub reflected, 54-56 voltage across its
//   impedance, 57-59 one step older, 60-62 Vc, 63-65 one step older.
// The coefficients are rebuilt from sx,sy,sz and the material every step, as
// in the reference.  Axis a = x,y,z has partners (j,k) = (y,z),(z,x),(x,y).
// ---------------------------------------------------------------------------
constexpr int kPmmState = 66;

struct PmmList {
  const int4 *pos;      // (x, y, z, output number or -1)
  const int2 *par_mat;  // (PML parameter row, 0-based; material, 1-based)
  double *state;        // [kPmmState][n]
  const double *sigma;  // [n_par][4]: sx, sy, sz, 0
  int n;
};

template <typename T>
__device__ __forceinline__ void pml_material_body(const MeshDev<T> &m, const PmmList &pl, int s, int rel_step) {
  const int t = *m.d_base + rel_step;
  const T *__restrict__ in = (t & 1) ? m.links0 : m.links1;
  T *__restrict__ out = (t & 1) ? m.links1 : m.links0;
  const long long P = m.plane;
  const int4 ps = pl.pos[s];
  const int2 pm = pl.par_mat[s];
  const int x = ps.x, y = ps.y, z = ps.z;
  const long long idx = (long long)(z + 1) * m.PxPy + (long long)(y + 1) * m.Px + x;
  const long long dy = m.Px, dz = m.PxPy;
  double V[12];
  V[Vy_xmin] = double(in[Vy_xmax * P + idx - 1]);
  V[Vz_xmin] = double(in[Vz_xmax * P + idx - 1]);
  V[Vy_xmax] = double(in[Vy_xmin * P + idx + 1]);
  V[Vz_xmax] = double(in[Vz_xmin * P + idx + 1]);
  V[Vx_ymin] = double(in[Vx_ymax * P + idx - dy]);
  V[Vz_ymin] = double(in[Vz_ymax * P + idx - dy]);
  V[Vx_ymax] = double(in[Vx_ymin * P + idx + dy]);
  V[Vz_ymax] = double(in[Vz_ymin * P + idx + dy]);
  V[Vx_zmin] = double(in[Vx_zmax * P + idx - dz]);
  V[Vy_zmin] = double(in[Vy_zmax * P + idx - dz]);
  V[Vx_zmax] = double(in[Vx_zmin * P + idx + dz]);
  V[Vy_zmax] = double(in[Vy_zmin * P + idx + dz]);

  const double *Pr = m.pml_par + (size_t)pm.x * 16;
  const double *Sg = pl.sigma + (size_t)pm.x * 4;
  const MatDev &mt = m.mats[pm.y - 1];
  const double dt = m.dt, Z0 = kZ0;
  const double Ys = mt.Ys_eps_f / kY0, Ge = mt.Ge / kY0, Zs = mt.Zs_mu_f, Rm = mt.Rm;
  const double sg[3] = {Sg[0], Sg[1], Sg[2]};
  const double ex[3] = {Pr[3], Pr[4], Pr[5]};
  double *S = pl.state;
  const int n = pl.n;
  auto ld = [&](int k) { return S[(size_t)k * n + s]; };
  auto st = [&](int k, double v) { S[(size_t)k * n + s] = v; };

  // STAGE 3
  V[Vynx] = V[Vynx] * ex[1]; V[Vypx] = V[Vypx] * ex[1];
  V[Vznx] = V[Vznx] * ex[2]; V[Vzpx] = V[Vzpx] * ex[2];
  V[Vxny] = V[Vxny] * ex[0]; V[Vxpy] = V[Vxpy] * ex[0];
  V[Vzny] = V[Vzny] * ex[2]; V[Vzpy] = V[Vzpy] * ex[2];
  V[Vxnz] = V[Vxnz] * ex[0]; V[Vxpz] = V[Vxpz] * ex[0];
  V[Vynz] = V[Vynz] * ex[1]; V[Vypz] = V[Vypz] * ex[1];

  double Vss[3], It_m1[3], It_m2[3], Vt[3], Vc[3], It[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    Vss[a] = -ld(51 + a);
    It_m1[a] = ld(30 + a);
    It_m2[a] = ld(33 + a);
  }
  // STAGE 4: stretched V with the capacitive stub
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const double sj = sg[(a + 1) % 3], sk = sg[(a + 2) % 3];
    const double GpY2 = (Ge + Ys) / 2.0;
    const double A0 = 8.0 + 4.0 * GpY2 + 2.0 * dt * (sj + sk) * (1.0 + GpY2) + dt * dt * sj * sk * GpY2;
    const double A1 = -2.0 * (8.0 + 4.0 * GpY2) + 2.0 * (dt * dt * sj * sk * GpY2);
    const double A2 = 8.0 + 4.0 * GpY2 - 2.0 * dt * (sj + sk) * (1.0 + GpY2) + dt * dt * sj * sk * GpY2;
    const double B0 = 4.0 + 2.0 * dt * sj, B1 = -8.0, B2 = 4.0 - 2.0 * dt * sj;
    const double C0 = 4.0 + 2.0 * dt * sk, C1 = -8.0, C2 = 4.0 - 2.0 * dt * sk;
    const double D0 = 4.0 * Ys + 2.0 * dt * (sj + sk) * Ys + 1.0 * (dt * dt * sj * sk * Ys);
    const double D1 = -8.0 * Ys + 2.0 * (dt * dt * sj * sk * Ys);
    const double D2 = 4.0 * Ys - 2.0 * dt * (sj + sk) * Ys + 1.0 * (dt * dt * sj * sk * Ys);
    // port pairs: B (x: Vznx,Vzpx  y: Vxny,Vxpy  z: Vynz,Vypz), C the others
    const int b0 = a == 0 ? Vznx : (a == 1 ? Vxny : Vynz), b1 = a == 0 ? Vzpx : (a == 1 ? Vxpy : Vypz);
    const int c0 = a == 0 ? Vynx : (a == 1 ? Vzny : Vxnz), c1 = a == 0 ? Vypx : (a == 1 ? Vzpy : Vxpz);
    const double Vos = ld(42 + a);
    Vt[a] = (1.0 / A0) * (B0 * (V[b0] + V[b1]) + C0 * (V[c0] + V[c1]) + D0 * (Vos) +
                          B1 * (ld(b0) + ld(b1)) + C1 * (ld(c0) + ld(c1)) + D1 * (ld(45 + a)) +
                          B2 * (ld(12 + b0) + ld(12 + b1)) + C2 * (ld(12 + c0) + ld(12 + c1)) + D2 * (ld(48 + a)) -
                          A1 * ld(24 + a) - A2 * ld(27 + a));
  }
  // STAGE 5: stretched I through the series impedance
  Vc[0] = V[Vypz] - V[Vzpy] - V[Vynz] + V[Vzny] - Vss[0];
  Vc[1] = V[Vzpx] - V[Vxpz] - V[Vznx] + V[Vxnz] - Vss[1];
  Vc[2] = V[Vxpy] - V[Vypx] - V[Vxny] + V[Vynx] - Vss[2];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const double sj = sg[(a + 1) % 3], sk = sg[(a + 2) % 3], sa = sg[a];
    const double ZpR = Zs + Rm;
    const double S0 = 16.0 * Z0 + 4.0 * ZpR + 2.0 * dt * (sj + sk) * (2.0 * Z0 + ZpR) + dt * dt * sj * sk * ZpR;
    const double S1 = -32.0 * Z0 - 8.0 * ZpR + 2.0 * dt * dt * sj * sk * ZpR;
    const double S2 = 16.0 * Z0 + 4.0 * ZpR - 2.0 * dt * (sj + sk) * (2.0 * Z0 + ZpR) + dt * dt * sj * sk * ZpR;
    const double T0 = 8.0 + 4.0 * dt * sa, T1 = -16.0, T2 = 8.0 - 4.0 * dt * sa;
    It[a] = (1.0 / S0) * (T0 * Vc[a] + T1 * ld(60 + a) + T2 * ld(63 + a) - S1 * It_m1[a] - S2 * It_m2[a]);
  }
  // series terms V_{ab}t, driven by the current of the third axis c; U uses
  // sigma_c, W sigma_b (order xy yx yz zy zx xz)
  double Vabt[6];
#pragma unroll
  for (int q = 0; q < 6; q++) {
    const int a = (q == 0 || q == 5) ? 0 : ((q == 1 || q == 2) ? 1 : 2);
    const int b = (q == 1 || q == 4) ? 0 : ((q == 0 || q == 3) ? 1 : 2);
    const int c = 3 - a - b;
    const double U0 = 2.0 + dt * sg[c], U1 = -2.0 + dt * sg[c];
    const double W0 = Z0 * (2.0 + dt * sg[b]), W1 = Z0 * (-2.0 + dt * sg[b]);
    Vabt[q] = (1.0 / U0) * (W0 * It[c] + W1 * It_m1[c] - U1 * ld(36 + q));
  }
  const double Vxyt = Vabt[0], Vyxt = Vabt[1], Vyzt = Vabt[2], Vzyt = Vabt[3], Vzxt = Vabt[4], Vxzt = Vabt[5];
  // STAGE 9: state for the next step
#pragma unroll
  for (int k = 0; k < 12; k++) {
    st(12 + k, ld(k));
    st(k, V[k]);
  }
#pragma unroll
  for (int a = 0; a < 3; a++) {
    st(27 + a, ld(24 + a));
    st(24 + a, Vt[a]);
    st(33 + a, It_m1[a]);
    st(30 + a, It[a]);
    st(63 + a, ld(60 + a));
    st(60 + a, Vc[a]);
  }
#pragma unroll
  for (int q = 0; q < 6; q++) st(36 + q, Vabt[q]);
  // STAGE 11: scattered pulses
  double R[12];
  R[Vynx] = Vt[0] - Vyxt - V[Vypx]; R[Vypx] = Vt[0] + Vyxt - V[Vynx];
  R[Vznx] = Vt[0] + Vzxt - V[Vzpx]; R[Vzpx] = Vt[0] - Vzxt - V[Vznx];
  R[Vzny] = Vt[1] - Vzyt - V[Vzpy]; R[Vzpy] = Vt[1] + Vzyt - V[Vzny];
  R[Vxny] = Vt[1] + Vxyt - V[Vxpy]; R[Vxpy] = Vt[1] - Vxyt - V[Vxny];
  R[Vxnz] = Vt[2] - Vxzt - V[Vxpz]; R[Vxpz] = Vt[2] + Vxzt - V[Vxnz];
  R[Vynz] = Vt[2] + Vyzt - V[Vypz]; R[Vypz] = Vt[2] - Vyzt - V[Vynz];
  // capacitive stub: reflect and keep the incident history
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const double Vos = ld(42 + a);
    st(42 + a, Vt[a] - Vos);
    st(48 + a, ld(45 + a));
    st(45 + a, Vos);
  }
  // inductive stub: voltage across the stub impedance, then its reflection
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const double sj = sg[(a + 1) % 3], sk = sg[(a + 2) % 3], sa = sg[a];
    const double P0 = 4.0 + 2.0 * dt * sa, P1 = -8.0, P2 = 4.0 - 2.0 * dt * sa;
    const double Q0 = 4.0 * Zs + 2.0 * dt * (sj + sk) * Zs + 1.0 * (dt * dt * sj * sk * Zs);
    const double Q1 = -8.0 * Zs + 2.0 * (dt * dt * sj * sk * Zs);
    const double Q2 = 4.0 * Zs - 2.0 * dt * (sj + sk) * Zs + 1.0 * (dt * dt * sj * sk * Zs);
    const double Vs = (1.0 / P0) * (Q0 * It[a] + Q1 * It_m1[a] + Q2 * It_m2[a] - P1 * ld(54 + a) - P2 * ld(57 + a));
    st(51 + a, (Vs + Vss[a]));
    st(57 + a, ld(54 + a));
    st(54 + a, Vs);
  }
  // STAGE 12: output
  if (ps.w >= 0) {
    const double dl = m.dl;
    const double f[6] = {-Vt[0] / dl, -Vt[1] / dl, -Vt[2] / dl, It[0] / dl, It[1] / dl, It[2] / dl};
    store_cell_out(m, t, ps.w, f);
  }
  // STAGE 13: half-cell loss on the scattered pulses, then the pulses leave
  R[Vynx] = R[Vynx] * ex[1]; R[Vypx] = R[Vypx] * ex[1];
  R[Vznx] = R[Vznx] * ex[2]; R[Vzpx] = R[Vzpx] * ex[2];
  R[Vxny] = R[Vxny] * ex[0]; R[Vxpy] = R[Vxpy] * ex[0];
  R[Vzny] = R[Vzny] * ex[2]; R[Vzpy] = R[Vzpy] * ex[2];
  R[Vxnz] = R[Vxnz] * ex[0]; R[Vxpz] = R[Vxpz] * ex[0];
  R[Vynz] = R[Vynz] * ex[1]; R[Vypz] = R[Vypz] * ex[1];
  T co[12];
#pragma unroll
  for (int p = 0; p < 12; p++) {
    co[p] = T(R[p]);
    out[p * P + idx] = co[p];
  }
  write_ghosts<T>(m, out, idx, x, y, z, co);
}

template <typename T>
__global__ void __launch_bounds__(128) tlm_pml_material_kernel(const MeshDev<T> m, const PmmList pl, int rel_step) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= pl.n) return;
  pml_material_body<T>(m, pl, s, rel_step);
}

// ---------------------------------------------------------------------------
// Special faces: Huygens excitation + face outputs, connect_normal_to_*.F90
// ---------------------------------------------------------------------------
// A dispersive thin layer after calculate_surface_material_filter_coefficients
// (MATERIALS/TLM_surface_materials.F90:225-280): per polarisation (x, y, z)
// and filter (Z11, Z12, Z21, Z22) the fast part f and the slow Z filter.
struct ThinLayerDev {
  double f[3][4];
  double a[3][4][kMaxOrder + 1], b[3][4][kMaxOrder + 1];
  int order[3][4];
};

struct FaceDev {
  const int4 *face;        // (x, y, z) 0-based of the + cell, dir 1..3
  const int2 *face_io;     // (exc index or -1, out index or -1)
  const double4 *hs;       // per special face: (offset, nx, ny, nz) when exc
  int n_faces;
  double Ei[3], Hi[3];
  double offset_min, c, dt, dl;
  const double *value_face;  // [n_timesteps] of the Huygens function
  int n_timesteps;
  double *face_field;      // [n_out_faces][2][6]
  const int2 *face_src;    // per special face: (Huygens patch 0/1, face point-source row or -1)
  const double *pt_field;  // [n_timesteps][n_pt_rows][2 sides][12] summed face sources (E, H, J, M)
  const int8_t *pt_type;   // [n_pt_rows][6] hard (0) / soft (1) source factor of E, H
  int n_pt_rows;
  const int8_t *mat;       // per special face: surface material 0 none, 1 PEC, 2 PMC, 3 thin layer, 4 free space
  const int *smat;         // per special face: signed thin-layer material (positive: reversed), 0 none
  const ThinLayerDev *tl;  // thin-layer materials
  double *tl_taps;         // per special face: [2 polarisations][4 filters][kMaxOrder] filter taps w(1..order)
};

// surface_material_update (MATERIALS/TLM_surface_materials.F90:535-697) for
// one polarisation of one face: the layer's two-port impedance matrix,
// fast parts plus the slow filters' responses, between the incident pulses
// Vli (from the cell below the face) and Vri (from the cell above), each
// side on the line impedance Z0; returns the total voltages Vl, Vr on the
// two sides and updates and time-shifts the four filters (taps w(1..order)
// at w + k * kMaxOrder).  The arithmetic is the reference's, in its order.
__device__ __forceinline__ void thin_layer_update(const ThinLayerDev &L, int pol, bool reverse, double *w,
                                                  double Vli, double Vri, double &Vl, double &Vr) {
  double slow[4];
  for (int k = 0; k < 4; k++) {  // evaluate_Zfilter with G = 0
    const int o = L.order[pol][k];
    const double *a = L.a[pol][k], *b = L.b[pol][k];
    const double *wk = w + k * kMaxOrder;
    double W0 = 0.0;
    for (int i = 1; i <= o; i++) W0 = W0 - b[i] * wk[i - 1];
    W0 = W0 / b[0];
    double F0 = 0.0;
    F0 = F0 + a[0] * W0;
    for (int i = 1; i <= o; i++) F0 = F0 + a[i] * wk[i - 1];
    slow[k] = F0;
  }
  const double Zl = kZ0, Zr = kZ0;
  const double Z1 = reverse ? Zr : Zl, Z2 = reverse ? Zl : Zr;
  const double U11 = Z1 + L.f[pol][0], U12 = L.f[pol][1], U21 = L.f[pol][2], U22 = Z2 + L.f[pol][3];
  const double det = U11 * U22 - U21 * U12;  // the host refuses layers for which it is zero
  const double V1i = reverse ? Vri : Vli, V2i = reverse ? Vli : Vri;
  const double rhs1 = 2.0 * V1i - slow[0] - slow[1];
  const double rhs2 = 2.0 * V2i - slow[2] - slow[3];
  const double i1 = (U22 * rhs1 - U12 * rhs2) / det;
  const double i2 = (-U21 * rhs1 + U11 * rhs2) / det;
  const double V1 = 2.0 * V1i - i1 * Z1;
  const double V2 = 2.0 * V2i - i2 * Z2;
  const double G[4] = {i1, i2, i1, i2};
  for (int k = 0; k < 4; k++) {  // evaluate_Zfilter with the port current, then timeshift_Zfilter
    const int o = L.order[pol][k];
    const double *b = L.b[pol][k];
    double *wk = w + k * kMaxOrder;
    double W0 = G[k];
    for (int i = 1; i <= o; i++) W0 = W0 - b[i] * wk[i - 1];
    W0 = W0 / b[0];
    for (int i = o - 1; i >= 1; i--) wk[i] = wk[i - 1];
    if (o > 0) wk[0] = W0;
  }
  Vl = reverse ? V2 : V1;
  Vr = reverse ? V1 : V2;
}

template <typename T>
__device__ __forceinline__ void face_body(const MeshDev<T> &m, const FaceDev &fd, int f, int rel_step);

template <typename T>
__global__ void tlm_face_kernel(const MeshDev<T> m, const FaceDev fd, int rel_step) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= fd.n_faces) return;
  face_body<T>(m, fd, f, rel_step);
}

// Outer-boundary Huygens surface (TLM_SOLVER/outer_boundary.F90:133-318):
// one thread per boundary face adds the surface's J, M to the two ghost
// slots that hold R times the boundary cell's reflected pulses (written by
// the cell kernels this step):
//   V - J dl Z0/2 + sg M dl/2 + R (-J dl Z0/2 - sg M dl/2)
// with the excitation value interpolated as for the connect faces
// (excitation.F90:645-690).
struct OuterHsDev {
  const int4 *face;      // (x, y, z) 0-based boundary cell, face code 1..6
  const double *offset;  // per face
  int n;
  double Ei[3], Hi[3];
  double offset_min, c, dt, dl;
  const double *value_face;  // [n_timesteps]
  int n_timesteps;
};

template <typename T>
__global__ void tlm_outer_huygens_kernel(const MeshDev<T> m, const OuterHsDev od, int rel_step) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= od.n) return;
  const int t = *m.d_base + rel_step;
  T *R = (t & 1) ? m.links1 : m.links0;
  const long long P = m.plane;
  const int4 fc = od.face[f];
  const int code = fc.w;
  const long long idx = (long long)(fc.z + 1) * m.PxPy + (long long)(fc.y + 1) * m.Px + fc.x;
  const double dt = od.dt;
  const double t_offset = (od.offset[f] - od.offset_min) / od.c;
  const double local_time = (double(t - 1)) * dt - t_offset;
  const int ts1 = (int)round(local_time / dt);
  const int ts2 = ts1 + 1;
  const double delta_t = local_time - double(ts1) * dt;
  const double v1 = (ts1 >= 1 && ts1 <= od.n_timesteps) ? od.value_face[ts1 - 1] : 0.0;
  const double v2 = (ts2 >= 1 && ts2 <= od.n_timesteps) ? od.value_face[ts2 - 1] : 0.0;
  const double value = v1 + delta_t * (v2 - v1) / dt;
  const int axis = (code - 1) % 3;
  const double nrm = code <= 3 ? -1.0 : 1.0;
  const double nx_ = axis == 0 ? nrm : 0.0, ny_ = axis == 1 ? nrm : 0.0, nz_ = axis == 2 ? nrm : 0.0;
  const double *Hi = od.Hi, *Ei = od.Ei;
  double Js[3], Ms[3];
  Js[0] = (ny_ * value * (Hi[2]) - nz_ * value * (Hi[1]));
  Js[1] = (nz_ * value * (Hi[0]) - nx_ * value * (Hi[2]));
  Js[2] = (nx_ * value * (Hi[1]) - ny_ * value * (Hi[0]));
  Ms[0] = -(ny_ * value * (Ei[2]) - nz_ * value * (Ei[1]));
  Ms[1] = -(nz_ * value * (Ei[0]) - nx_ * value * (Ei[2]));
  Ms[2] = -(nx_ * value * (Ei[1]) - ny_ * value * (Ei[0]));
  // ghost slot of each tangential port, its J and M components, and the
  // sign of M on the first port (the second port takes the opposite sign)
  long long g0, g1;
  int j0, m0, j1, m1;
  double s0;
  const long long dy = m.Px, dz = m.PxPy;
  switch (code) {
    case 1: g0 = Vy_xmax * P + idx - 1; g1 = Vz_xmax * P + idx - 1; j0 = 1; m0 = 2; j1 = 2; m1 = 1; s0 = -1.0; break;
    case 2: g0 = Vx_ymax * P + idx - dy; g1 = Vz_ymax * P + idx - dy; j0 = 0; m0 = 2; j1 = 2; m1 = 0; s0 = 1.0; break;
    case 3: g0 = Vx_zmax * P + idx - dz; g1 = Vy_zmax * P + idx - dz; j0 = 0; m0 = 1; j1 = 1; m1 = 0; s0 = -1.0; break;
    case 4: g0 = Vy_xmin * P + idx + 1; g1 = Vz_xmin * P + idx + 1; j0 = 1; m0 = 2; j1 = 2; m1 = 1; s0 = 1.0; break;
    case 5: g0 = Vx_ymin * P + idx + dy; g1 = Vz_ymin * P + idx + dy; j0 = 0; m0 = 2; j1 = 2; m1 = 0; s0 = -1.0; break;
    default: g0 = Vx_zmin * P + idx + dz; g1 = Vy_zmin * P + idx + dz; j0 = 0; m0 = 1; j1 = 1; m1 = 0; s0 = 1.0; break;
  }
  const double Rf = double(m.R[code <= 3 ? 2 * (code - 1) : 2 * (code - 4) + 1]);
  const double dl = od.dl, Z0 = kZ0;
  const double v0 = double(R[g0]), w0 = double(R[g1]);
  R[g0] = T(v0 - Js[j0] * dl * Z0 / 2.0 + s0 * Ms[m0] * dl / 2.0 + Rf * (-Js[j0] * dl * Z0 / 2.0 - s0 * Ms[m0] * dl / 2.0));
  R[g1] = T(w0 - Js[j1] * dl * Z0 / 2.0 - s0 * Ms[m1] * dl / 2.0 + Rf * (-Js[j1] * dl * Z0 / 2.0 + s0 * Ms[m1] * dl / 2.0));
}

// face_output_points (output_points.F90:255-444): one thread per face output
// point copies its side and component of face_output_field, after connect.
struct FaceProbeDev {
  const int4 *probe;  // (output face 0-based, side 0/1, component 0..5, 0)
  double *rec;        // [n_timesteps][n]
  int n;
};

__global__ void tlm_face_probe_kernel(const FaceProbeDev pd, const double *face_field, const int *d_base,
                                      int rel_step) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= pd.n) return;
  const int t = *d_base + rel_step;
  const int4 pr = pd.probe[q];
  pd.rec[(size_t)(t - 1) * pd.n + q] = face_field[(size_t)pr.x * 12 + pr.y * 6 + pr.z];
}

template <typename T>
__device__ __forceinline__ void face_body(const MeshDev<T> &m, const FaceDev &fd, int f, int rel_step) {
  const int t = *m.d_base + rel_step;
  T *R = (t & 1) ? m.links1 : m.links0;  // R_t just written by the cell kernel
  const long long P = m.plane;
  const int4 fc = fd.face[f];
  const int2 io = fd.face_io[f];
  const int dir = fc.w;
  const long long ip = (long long)(fc.z + 1) * m.PxPy + (long long)(fc.y + 1) * m.Px + fc.x;  // + cell
  const long long step = dir == 1 ? 1 : (dir == 2 ? (long long)m.Px : m.PxPy);
  const long long im = ip - step;  // - cell
  int pmin1, pmax1, pmin2, pmax2;
  if (dir == 1) { pmin1 = Vy_xmin; pmax1 = Vy_xmax; pmin2 = Vz_xmin; pmax2 = Vz_xmax; }
  else if (dir == 2) { pmin1 = Vx_ymin; pmax1 = Vx_ymax; pmin2 = Vz_ymin; pmax2 = Vz_ymax; }
  else { pmin1 = Vx_zmin; pmax1 = Vx_zmax; pmin2 = Vy_zmin; pmax2 = Vy_zmax; }
  // reflected pulses at the face: a = from the + cell (its min port), b = from the - cell
  const double a1 = double(R[pmin1 * P + ip]), b1 = double(R[pmax1 * P + im]);
  const double a2 = double(R[pmin2 * P + ip]), b2 = double(R[pmax2 * P + im]);
  double A_min = a1 + b1, A_max = A_min;
  double B_min = a2 + b2, B_max = B_min;
  const int mat = fd.mat[f];
  if (mat == 1) {  // PEC sheet, connect_normal_to_x.F90:36-40: each side reflects with -1
    A_min = 0.0; A_max = 0.0; B_min = 0.0; B_max = 0.0;
  } else if (mat == 2) {  // PMC sheet, connect_normal_to_x.F90:41-45: each side reflects with +1
    A_min = 2.0 * a1; A_max = 2.0 * b1; B_min = 2.0 * a2; B_max = 2.0 * b2;
  } else if (mat == 3) {  // thin layer, connect_normal_to_x.F90:268-282 (y, z analogues)
    const int sm = fd.smat[f];
    const ThinLayerDev &L = fd.tl[(sm > 0 ? sm : -sm) - 1];
    const int pol1 = dir == 1 ? 1 : 0, pol2 = dir == 3 ? 1 : 2;  // x faces: y, z; y faces: x, z; z faces: x, y
    double *w = fd.tl_taps + (size_t)f * 8 * kMaxOrder;
    thin_layer_update(L, pol1, sm > 0, w, b1, a1, A_max, A_min);
    thin_layer_update(L, pol2, sm > 0, w + 4 * kMaxOrder, b2, a2, B_max, B_min);
  }  // 0 and 4 (a free-space surface material): the plain sum
  if (io.x >= 0) {
    // face_excitation_field / face_excitation_type of this face, side 1
    // (min) and side 2 (max): point sources on both sides
    // (excitation_points.F90:286-323), one-sided or two-sided excitation
    // surfaces (excitation_surfaces.F90:218-275), then the Huygens J, M on
    // both sides (huygens_surface.F90:734-848)
    const int2 src = fd.face_src[f];
    double fld[2][6], Js[2][3], Ms[2][3];
    double hsf[6] = {1.0, 1.0, 1.0, 1.0, 1.0, 1.0};
#pragma unroll
    for (int sd = 0; sd < 2; sd++) {
#pragma unroll
      for (int k = 0; k < 6; k++) fld[sd][k] = 0.0;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        Js[sd][k] = 0.0;
        Ms[sd][k] = 0.0;
      }
    }
    if (src.y >= 0) {
      const double *pf = fd.pt_field + ((size_t)(t - 1) * fd.n_pt_rows + src.y) * 24;
      const int8_t *ty = fd.pt_type + (size_t)src.y * 6;
#pragma unroll
      for (int sd = 0; sd < 2; sd++) {
#pragma unroll
        for (int k = 0; k < 6; k++) fld[sd][k] = pf[sd * 12 + k];
#pragma unroll
        for (int k = 0; k < 3; k++) {
          Js[sd][k] = pf[sd * 12 + 6 + k];
          Ms[sd][k] = pf[sd * 12 + 9 + k];
        }
      }
#pragma unroll
      for (int k = 0; k < 6; k++) hsf[k] = double(ty[k]);
    }
    if (src.x) {
      // get_interpolated_excitation_value (excitation.F90:645-690)
      const double4 h = fd.hs[f];
      const double dt = fd.dt;
      const double t_offset = (h.x - fd.offset_min) / fd.c;
      const double local_time = (double(t - 1)) * dt - t_offset;
      const int ts1 = (int)round(local_time / dt);
      const int ts2 = ts1 + 1;
      const double delta_t = local_time - double(ts1) * dt;
      const double v1 = (ts1 >= 1 && ts1 <= fd.n_timesteps) ? fd.value_face[ts1 - 1] : 0.0;
      const double v2 = (ts2 >= 1 && ts2 <= fd.n_timesteps) ? fd.value_face[ts2 - 1] : 0.0;
      const double value = v1 + delta_t * (v2 - v1) / dt;
      const double nx_ = h.y, ny_ = h.z, nz_ = h.w;
      const double *Hi = fd.Hi, *Ei = fd.Ei;
      const double j0 = (ny_ * value * (Hi[2]) - nz_ * value * (Hi[1]));
      const double j1 = (nz_ * value * (Hi[0]) - nx_ * value * (Hi[2]));
      const double j2 = (nx_ * value * (Hi[1]) - ny_ * value * (Hi[0]));
      const double m0 = -(ny_ * value * (Ei[2]) - nz_ * value * (Ei[1]));
      const double m1 = -(nz_ * value * (Ei[0]) - nx_ * value * (Ei[2]));
      const double m2 = -(nx_ * value * (Ei[1]) - ny_ * value * (Ei[0]));
#pragma unroll
      for (int sd = 0; sd < 2; sd++) {
        Js[sd][0] = Js[sd][0] + j0;
        Js[sd][1] = Js[sd][1] + j1;
        Js[sd][2] = Js[sd][2] + j2;
        Ms[sd][0] = Ms[sd][0] + m0;
        Ms[sd][1] = Ms[sd][1] + m1;
        Ms[sd][2] = Ms[sd][2] + m2;
      }
    }
    const double dl = fd.dl, Z0 = kZ0;
    const double *fn = fld[0], *fx = fld[1], *Jn = Js[0], *Jx = Js[1], *Mn = Ms[0], *Mx = Ms[1];
    // connect_normal_to_{x,y,z}.F90: the side-1 source types act on both sides
    if (dir == 1) {  // connect_normal_to_x.F90:301-305
      A_min = A_min * hsf[1] - fn[1] * dl - fn[5] * Z0 * dl + Jn[1] * dl * Z0 / 2.0 + Mn[2] * dl / 2.0;
      A_max = A_max * hsf[1] - fx[1] * dl + fx[5] * Z0 * dl + Jx[1] * dl * Z0 / 2.0 - Mx[2] * dl / 2.0;
      B_min = B_min * hsf[2] - fn[2] * dl + fn[4] * Z0 * dl + Jn[2] * dl * Z0 / 2.0 - Mn[1] * dl / 2.0;
      B_max = B_max * hsf[2] - fx[2] * dl - fx[4] * Z0 * dl + Jx[2] * dl * Z0 / 2.0 + Mx[1] * dl / 2.0;
    } else if (dir == 2) {  // connect_normal_to_y.F90:304-308
      A_min = A_min * hsf[0] - fn[0] * dl + fn[5] * Z0 * dl + Jn[0] * dl * Z0 / 2.0 - Mn[2] * dl / 2.0;
      A_max = A_max * hsf[0] - fx[0] * dl - fx[5] * Z0 * dl + Jx[0] * dl * Z0 / 2.0 + Mx[2] * dl / 2.0;
      B_min = B_min * hsf[2] - fn[2] * dl - fn[3] * Z0 * dl + Jn[2] * dl * Z0 / 2.0 + Mn[0] * dl / 2.0;
      B_max = B_max * hsf[2] - fx[2] * dl + fx[3] * Z0 * dl + Jx[2] * dl * Z0 / 2.0 - Mx[0] * dl / 2.0;
    } else {  // connect_normal_to_z.F90:302-306
      A_min = A_min * hsf[0] - fn[0] * dl - fn[4] * Z0 * dl + Jn[0] * dl * Z0 / 2.0 + Mn[1] * dl / 2.0;
      A_max = A_max * hsf[0] - fx[0] * dl + fx[4] * Z0 * dl + Jx[0] * dl * Z0 / 2.0 - Mx[1] * dl / 2.0;
      B_min = B_min * hsf[1] - fn[1] * dl + fn[3] * Z0 * dl + Jn[1] * dl * Z0 / 2.0 - Mn[0] * dl / 2.0;
      B_max = B_max * hsf[1] - fx[1] * dl - fx[3] * Z0 * dl + Jx[1] * dl * Z0 / 2.0 + Mx[0] * dl / 2.0;
    }
  }
  // new incident pulses: + cell pulls its min port from the - cell's max-port
  // slot, the - cell pulls its max port from the + cell's min-port slot
  const double inc_p1 = A_min - a1, inc_m1 = A_max - b1;
  const double inc_p2 = B_min - a2, inc_m2 = B_max - b2;
  R[pmax1 * P + im] = T(inc_p1);
  R[pmin1 * P + ip] = T(inc_m1);
  R[pmax2 * P + im] = T(inc_p2);
  R[pmin2 * P + ip] = T(inc_m2);
  if (io.y >= 0) {
    const double dl = fd.dl, Z0 = kZ0;
    double *fo = fd.face_field + (size_t)io.y * 12;
    for (int side = 0; side < 2; side++) {
      // side 1: positive = incident into + cell, negative = reflected from + cell
      const double pa = side ? b1 : inc_p1, na = side ? inc_m1 : a1;
      const double pb = side ? b2 : inc_p2, nb = side ? inc_m2 : a2;
      double *fl = fo + side * 6;
      if (dir == 1) {
        fl[0] = 0.0; fl[1] = -(pa + na) / dl; fl[2] = -(pb + nb) / dl;
        fl[3] = 0.0; fl[4] = (pb - nb) / (Z0 * dl); fl[5] = -(pa - na) / (Z0 * dl);
      } else if (dir == 2) {
        fl[0] = -(pa + na) / dl; fl[1] = 0.0; fl[2] = -(pb + nb) / dl;
        fl[3] = -(pb - nb) / (Z0 * dl); fl[4] = 0.0; fl[5] = (pa - na) / (Z0 * dl);
      } else {
        fl[0] = -(pa + na) / dl; fl[1] = -(pb + nb) / dl; fl[2] = 0.0;
        fl[3] = (pb - nb) / (Z0 * dl); fl[4] = -(pa - na) / (Z0 * dl); fl[5] = 0.0;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// FP64 DFT accumulation, frequency_output_surfaces.F90:343-410
// ---------------------------------------------------------------------------
// Time-domain output surfaces, face_output_surfaces (output_surfaces.F90:
// 601-760): on the output steps of a surface (first..last every interval)
// each face's value is written to row (t - first) / interval of the
// surface's history.  The face code (after the side flip) gives the side of
// face_output_field (1 on a min face, 2 on a max face) and the normal n
// (+1 on a min face, -1 on a max face); with both_sides the two sides are
// field and field2.  Components: 1..6 field(c); 7..9 J = n x H(field) -
// n x H(field2); 13 |E|, 14 |H| of field; 15 |J|.
struct OSurfDev {
  int4 gate;      // first, last, interval, component
  int both, n_faces;
  long long off;  // first value of the surface in the history
};
struct OutSurfDev {
  int n_entries;
  const int2 *entry;         // (surface, face output 0-based)
  const int2 *pos;           // (face code 1..6, index within the surface)
  const OSurfDev *surf;
  const double *face_field;  // [n_out_faces][2][6]
  double *hist;
};

__global__ void tlm_output_surface_kernel(const OutSurfDev d, const int *d_base, int rel_step) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n_entries) return;
  const int t = *d_base + rel_step;
  const int2 e = d.entry[k];
  const OSurfDev sf = d.surf[e.x];
  const int4 g = sf.gate;
  if (t < g.x || t > g.y || (t - g.x) % g.z != 0) return;
  const int2 q = d.pos[k];
  const int code = q.x;
  const int side = code <= 3 ? 0 : 1;
  double normx = 0.0, normy = 0.0, normz = 0.0;
  if (code == 1) normx = 1.0; else if (code == 4) normx = -1.0;
  else if (code == 2) normy = 1.0; else if (code == 5) normy = -1.0;
  else if (code == 3) normz = 1.0; else normz = -1.0;
  const double *ff = d.face_field + (size_t)e.y * 12;
  double f[6], f2[6];
#pragma unroll
  for (int c = 0; c < 6; c++) {
    f[c] = sf.both ? ff[c] : ff[side * 6 + c];
    f2[c] = sf.both ? ff[6 + c] : 0.0;
  }
  // field indices: Ex Ey Ez Hx Hy Hz = 0..5
  const double Jsx = (normy * f[5] - normz * f[4]) - (normy * f2[5] - normz * f2[4]);
  const double Jsy = (normz * f[3] - normx * f[5]) - (normz * f2[3] - normx * f2[5]);
  const double Jsz = (normx * f[4] - normy * f[3]) - (normx * f2[4] - normy * f2[3]);
  double v;
  const int comp = g.w;
  if (comp <= 6) v = f[comp - 1];
  else if (comp == 7) v = Jsx;
  else if (comp == 8) v = Jsy;
  else if (comp == 9) v = Jsz;
  else if (comp == 13) v = sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
  else if (comp == 14) v = sqrt(f[3] * f[3] + f[4] * f[4] + f[5] * f[5]);
  else v = sqrt(Jsx * Jsx + Jsy * Jsy + Jsz * Jsz);
  d.hist[sf.off + (long long)((t - g.x) / g.z) * sf.n_faces + q.y] = v;
}

// Time-domain far field for the RCS surface, face_output_rcs
// (RCS_surfaces.F90:386-560).  Every step each face adds its contribution
// to the far-field time bin
//   point = INT(npc * (-(K.x) + time c0) / dl) - offset   (kept when 1..n_points),
// time the face-output time (timestep-1) dt + dt/2, from its fields on its
// side of face_output_field: Js = n x H, Ms = -(n x E), n = +1 on a min
// face and -1 on a max face; N, L = (Js, Ms) projected on theta and phi
// times dA / (4 pi); Etheta = -(Lphi + Z0 Ntheta), Ephi = Ltheta - Z0 Nphi,
// Htheta = Nphi - Ltheta / Z0, Hphi = -(Ntheta + Lphi / Z0).
// The host sorts the faces by K.x, so INT(...) does not increase along the
// list and the faces of one bin form one run; the first face of each run
// adds the run's contributions in list order.  The bin arithmetic is
// rounded step by step (no contraction) so that it matches the oracle's.
struct RcsDev {
  int n_faces, n_points, npc, offset;
  double ct, st, cp, sp, dA, four_pi, dl;
  const int2 *face;          // (face output 0-based, face code 1..6), sorted by K.x
  const double *dist;        // K.x of each face, ascending
  const double *tc0;         // [n_timesteps]: time * c0 at the face outputs
  const double *face_field;  // [n_out_faces][2][6]
  double *acc;               // [4][n_points]: Etheta, Ephi, Htheta, Hphi
};

__device__ __forceinline__ int rcs_point(const RcsDev &d, int i, double tc0) {
  const double a = __dadd_rn(-d.dist[i], tc0);
  const double b = __ddiv_rn(__dmul_rn((double)d.npc, a), d.dl);
  return (int)b - d.offset;  // INT truncates toward zero, as C does
}

__global__ void tlm_rcs_kernel(const RcsDev d, const int *d_base, int rel_step) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n_faces) return;
  const int t = *d_base + rel_step;
  const double tc0 = d.tc0[t - 1];
  const int p = rcs_point(d, i, tc0);
  if (i > 0 && rcs_point(d, i - 1, tc0) == p) return;  // not the first face of its run
  if (p < 1 || p > d.n_points) return;
  const size_t np = (size_t)d.n_points;
  double et = d.acc[p - 1], ep = d.acc[np + p - 1], ht = d.acc[2 * np + p - 1], hp = d.acc[3 * np + p - 1];
  for (int j = i; j < d.n_faces; j++) {
    if (j > i && rcs_point(d, j, tc0) != p) break;
    const int2 fc = d.face[j];
    const int side = fc.y <= 3 ? 0 : 1;
    double normx = 0.0, normy = 0.0, normz = 0.0;
    if (fc.y == 1) normx = 1.0; else if (fc.y == 4) normx = -1.0;
    else if (fc.y == 2) normy = 1.0; else if (fc.y == 5) normy = -1.0;
    else if (fc.y == 3) normz = 1.0; else normz = -1.0;
    const double *f = d.face_field + (size_t)fc.x * 12 + side * 6;
    const double Jsx = normy * f[5] - normz * f[4], Jsy = normz * f[3] - normx * f[5], Jsz = normx * f[4] - normy * f[3];
    const double Msx = -(normy * f[2] - normz * f[1]), Msy = -(normz * f[0] - normx * f[2]);
    const double Msz = -(normx * f[1] - normy * f[0]);
    const double Nt = (Jsx * d.ct * d.cp + Jsy * d.ct * d.sp - Jsz * d.st) * d.dA / d.four_pi;
    const double Np = (-Jsx * d.sp + Jsy * d.cp) * d.dA / d.four_pi;
    const double Lt = (Msx * d.ct * d.cp + Msy * d.ct * d.sp - Msz * d.st) * d.dA / d.four_pi;
    const double Lp = (-Msx * d.sp + Msy * d.cp) * d.dA / d.four_pi;
    et = et + (-(Lp + kZ0 * Nt));
    ep = ep + (Lt - kZ0 * Np);
    ht = ht + (Np - Lt / kZ0);
    hp = hp + (-(Nt + Lp / kZ0));
  }
  d.acc[p - 1] = et; d.acc[np + p - 1] = ep; d.acc[2 * np + p - 1] = ht; d.acc[3 * np + p - 1] = hp;
}

// Time-domain output volumes on their output steps (first..last every
// interval), from the current-step cell output rows:
//   kind 0, cell_output_volumes (output_volumes.F90:20-140): each cell's
//     field(component) into row (t - first) / interval of the volume's history;
//   kind 1, cell_output_volume_averages (output_volume_averages.F90): the
//     sum over the cells divided by their number;
//   kind 2, cell_output_volume_peak (output_volume_peak.F90): the largest
//     |field(component)|, from 0;
// kinds 1 and 2 write 0 when |value| < 1e-30.  One block per volume; the
// sum is taken in a fixed order (strided partial sums, then a fixed tree),
// so it is the same on every run and in a batch.
struct OVolDev {
  int4 gate;      // first, last, interval, component 1..6
  int kind, n_cells, cell0;
  long long off;  // first value of the volume in the history
};
struct OutVolDev {
  int n_vol;
  const OVolDev *vol;
  const int *cells;          // output cell 0-based, volume after volume
  const double *cell_cur;    // [n_out][6]
  double *hist;
};
constexpr int kOutVolThreads = 256;

__global__ void __launch_bounds__(kOutVolThreads) tlm_output_volume_kernel(const OutVolDev d, const int *d_base,
                                                                             int rel_step) {
  __shared__ double red[kOutVolThreads];
  const OVolDev v = d.vol[blockIdx.x];
  const int t = *d_base + rel_step;
  const int4 g = v.gate;
  if (t < g.x || t > g.y || (t - g.x) % g.z != 0) return;  // uniform over the block
  const long long row = (t - g.x) / g.z;
  const int tid = threadIdx.x;
  const int *cells = d.cells + v.cell0;
  if (v.kind == 0) {
    for (int k = tid; k < v.n_cells; k += kOutVolThreads)
      d.hist[v.off + row * v.n_cells + k] = d.cell_cur[(size_t)cells[k] * 6 + (g.w - 1)];
    return;
  }
  double a = 0.0;
  for (int k = tid; k < v.n_cells; k += kOutVolThreads) {
    const double x = d.cell_cur[(size_t)cells[k] * 6 + (g.w - 1)];
    a = v.kind == 1 ? a + x : fmax(a, fabs(x));
  }
  red[tid] = a;
  __syncthreads();
  for (int w = kOutVolThreads / 2; w > 0; w >>= 1) {
    if (tid < w) red[tid] = v.kind == 1 ? red[tid] + red[tid + w] : fmax(red[tid], red[tid + w]);
    __syncthreads();
  }
  if (tid == 0) {
    double r = red[0];
    if (v.kind == 1) r = v.n_cells ? r / (double)v.n_cells : 0.0;
    if (fabs(r) < 1e-30) r = 0.0;
    d.hist[v.off + row] = r;
  }
}

// SAR volumes, cell_output_SAR_volumes (SAR_volumes.F90:257-330): every
// step each cell accumulates E_c += exp(-j 2 pi f time) * E_c(t) * dt,
// c = x, y, z, at the cell-output time (timestep-1) dt, for write_SAR_volumes
// to turn into SAR afterwards.  One thread per (volume, cell) entry.
struct SarDev {
  int n_entries, n_vol;
  double dt;
  const int2 *entry;       // (volume, output cell 0-based)
  const double2 *phasor;   // [n_timesteps][n_vol]: exp(-j 2 pi f (timestep-1) dt)
  const double *cell_cur;  // [n_out][6]
  double2 *acc;            // [n_entries][3]
};

__global__ void tlm_sar_kernel(const SarDev d, const int *d_base, int rel_step) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n_entries) return;
  const int t = *d_base + rel_step;
  const int2 e = d.entry[k];
  const double2 p = d.phasor[(size_t)(t - 1) * d.n_vol + e.x];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const double v = d.cell_cur[(size_t)e.y * 6 + c];
    double2 a = d.acc[(size_t)k * 3 + c];
    a.x = a.x + p.x * v * d.dt;
    a.y = a.y + p.y * v * d.dt;
    d.acc[(size_t)k * 3 + c] = a;
  }
}

// Frequency-domain power surfaces, face_output_frequency_domain_power_surfaces
// (frequency_domain_power_surfaces.F90:287-420): every step each face adds
// E1, E2, H1, H2 times exp(-j 2 pi f time), at the face-output time, where
// (E1, E2, H1, H2) are the tangential fields on the face's side: (Ey, Ez,
// Hy, Hz) on x faces, (Ez, Ex, Hz, Hx) on y faces, (Ex, Ey, Hx, Hy) on z
// faces.  One thread per (surface and frequency, face) entry.
struct PowerSurfDev {
  int n_entries, n_ps;
  const int4 *entry;         // (surface-frequency, face output 0-based, face code 1..6, 0)
  const double2 *phasor;     // [n_timesteps][n_ps]
  const double *face_field;  // [n_out_faces][2][6]
  double2 *acc;              // [n_entries][4]
};

__global__ void tlm_power_surface_kernel(const PowerSurfDev d, const int *d_base, int rel_step) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n_entries) return;
  const int t = *d_base + rel_step;
  const int4 e = d.entry[k];
  const int axis = (e.z - 1) % 3, side = e.z <= 3 ? 0 : 1;
  const double *f = d.face_field + (size_t)e.y * 12 + side * 6;
  const int c1 = axis == 0 ? 1 : (axis == 1 ? 2 : 0), c2 = axis == 0 ? 2 : (axis == 1 ? 0 : 1);
  const double v[4] = {f[c1], f[c2], f[3 + c1], f[3 + c2]};
  const double2 p = d.phasor[(size_t)(t - 1) * d.n_ps + e.x];
#pragma unroll
  for (int c = 0; c < 4; c++) {
    double2 a = d.acc[(size_t)k * 4 + c];
    a.x = a.x + v[c] * p.x;
    a.y = a.y + v[c] * p.y;
    d.acc[(size_t)k * 4 + c] = a;
  }
}

// Mode outputs, Mode_output (output_modes.F90:546-620): every step each
// mode's value is the sum over its faces of face_output_field(side, component)
// times the mode field at the face, 0 when below 1e-30 in magnitude.  One
// block per mode, the sum in a fixed order (strided partial sums, then a
// fixed tree).
struct ModeDev {
  int n_modes;
  const int4 *mode;          // (first face entry, n_faces, component 1..6, 0)
  const int2 *face;          // (face output 0-based, face code 1..6)
  const double *weight;      // mode field per face entry
  const double *face_field;  // [n_out_faces][2][6]
  double *hist;              // [n_timesteps][n_modes]
};

__global__ void __launch_bounds__(kOutVolThreads) tlm_mode_kernel(const ModeDev d, const int *d_base, int rel_step) {
  __shared__ double red[kOutVolThreads];
  const int4 md = d.mode[blockIdx.x];
  const int t = *d_base + rel_step;
  const int tid = threadIdx.x;
  double a = 0.0;
  for (int k = tid; k < md.y; k += kOutVolThreads) {
    const int2 fc = d.face[md.x + k];
    const int side = fc.y <= 3 ? 0 : 1;
    a = a + d.face_field[(size_t)fc.x * 12 + side * 6 + (md.z - 1)] * d.weight[md.x + k];
  }
  red[tid] = a;
  __syncthreads();
  for (int w = kOutVolThreads / 2; w > 0; w >>= 1) {
    if (tid < w) red[tid] = red[tid] + red[tid + w];
    __syncthreads();
  }
  if (tid == 0) {
    double r = red[0];
    if (fabs(r) < 1e-30) r = 0.0;
    d.hist[(size_t)(t - 1) * d.n_modes + blockIdx.x] = r;
  }
}

// Frequency-domain output volumes, frequency_output_volumes.F90:309-390:
// on the output steps of a volume (get_output_flag, output.F90:564-598:
// first <= t <= last and (t - first) mod interval == 0),
//   value(cell) += cell_output_field(cell, component) * exp(-j 2 pi f time),
// time = (timestep-1) dt, the time of the cell outputs.  One thread per
// (volume, cell) entry; it reads the current-step row of its output cell.
struct VolDftDev {
  int n_entries, n_vol;
  const int2 *entry;       // (volume, output cell 0-based)
  const int4 *gate;        // per volume: (first, last, interval, component 1..6)
  const double2 *phasor;   // [n_timesteps][n_vol]: exp(-j 2 pi f (timestep-1) dt)
  const double *cell_cur;  // [n_out][6]
  double2 *acc;            // [n_entries]
};

__global__ void tlm_volume_dft_kernel(const VolDftDev d, const int *d_base, int rel_step) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n_entries) return;
  const int t = *d_base + rel_step;
  const int2 e = d.entry[k];
  const int4 g = d.gate[e.x];
  if (t < g.x || t > g.y || (t - g.x) % g.z != 0) return;
  const double v = d.cell_cur[(size_t)e.y * 6 + (g.w - 1)];
  const double2 p = d.phasor[(size_t)(t - 1) * d.n_vol + e.x];
  double2 a = d.acc[k];
  a.x = a.x + v * p.x;
  a.y = a.y + v * p.y;
  d.acc[k] = a;
}

struct DftDev {
  int n_entries, n_dft;
  const int4 *entry;        // (surface, out face index, face code 1..6, component 1..9)
  const double2 *phasor;    // [n_timesteps][n_dft] exp(-j 2 pi f t)
  const double *face_field; // [n_out_faces][2][6]
  double2 *acc;             // [n_entries]
};

__device__ __forceinline__ void dft_body(const DftDev &d, const int *d_base, int k, int rel_step);

__global__ void tlm_dft_kernel(const DftDev d, const int *d_base, int rel_step) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n_entries) return;
  dft_body(d, d_base, k, rel_step);
}

__device__ __forceinline__ void dft_body(const DftDev &d, const int *d_base, int k, int rel_step) {
  const int t = *d_base + rel_step;
  const int4 en = d.entry[k];
  const int face = en.z;
  const int side = face <= 3 ? 0 : 1;
  double normx = 0, normy = 0, normz = 0;
  if (face == 1) normx = 1; else if (face == 4) normx = -1;
  else if (face == 2) normy = 1; else if (face == 5) normy = -1;
  else if (face == 3) normz = 1; else normz = -1;
  const double *fl = d.face_field + (size_t)en.y * 12 + side * 6;
  double value;
  if (en.w <= 6) value = fl[en.w - 1];
  else if (en.w == 7) value = (normy * fl[5] - normz * fl[4]);
  else if (en.w == 8) value = (normz * fl[3] - normx * fl[5]);
  else value = (normx * fl[4] - normy * fl[3]);
  const double2 ph = d.phasor[(size_t)(t - 1) * d.n_dft + en.x];
  double2 a = d.acc[k];
  a.x = a.x + value * ph.x;
  a.y = a.y + value * ph.y;
  d.acc[k] = a;
}

// face_output_far_field (far_field_surfaces.F90:252-351): one thread per
// (surface, face) entry accumulates J += e^{-jwt} dt (n x H) and
// M -= e^{-jwt} dt (n x E) from the entry's side of face_output_field.
struct FarFieldDev {
  int n_entries, n_ff;
  const int4 *entry;        // (surface, out face index, face code 1..6, 0)
  const double2 *phasor;    // [n_timesteps][n_ff] exp(-j 2 pi f t) dt
  const double *face_field; // [n_out_faces][2][6]
  double2 *acc;             // [n_entries][6]: Jx, Jy, Jz, Mx, My, Mz
};

__global__ void tlm_far_field_kernel(const FarFieldDev d, const int *d_base, int rel_step) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n_entries) return;
  const int t = *d_base + rel_step;
  const int4 en = d.entry[k];
  const int face = en.z;
  const int side = face <= 3 ? 0 : 1;
  double normx = 0, normy = 0, normz = 0;
  if (face == 1) normx = 1; else if (face == 4) normx = -1;
  else if (face == 2) normy = 1; else if (face == 5) normy = -1;
  else if (face == 3) normz = 1; else normz = -1;
  const double *fl = d.face_field + (size_t)en.y * 12 + side * 6;
  double v[6];
  v[0] = (normy * fl[5] - normz * fl[4]);
  v[1] = (normz * fl[3] - normx * fl[5]);
  v[2] = (normx * fl[4] - normy * fl[3]);
  v[3] = (normy * fl[2] - normz * fl[1]);
  v[4] = (normz * fl[0] - normx * fl[2]);
  v[5] = (normx * fl[1] - normy * fl[0]);
  const double2 ph = d.phasor[(size_t)(t - 1) * d.n_ff + en.x];
  double2 *a = d.acc + (size_t)k * 6;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    double2 j = a[c], m = a[3 + c];
    j.x = j.x + ph.x * v[c];
    j.y = j.y + ph.y * v[c];
    m.x = m.x - ph.x * v[3 + c];
    m.y = m.y - ph.y * v[3 + c];
    a[c] = j;
    a[3 + c] = m;
  }
}

__global__ void tlm_advance_base(int *d_base, int n) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *d_base += n;
}

// ---------------------------------------------------------------------------
// Batched execution: many meshes (of one precision) advanced together.  Each
// kernel walks a block list of (mesh, first item) pairs; block b does items
// first..first+blockDim-1 of mesh b.x.  Per-mesh tables live in device arrays.
// ---------------------------------------------------------------------------
template <typename T>
struct BatchDev {
  const MeshDev<T> *meshes;
  const PmlList *pml;
  const FaceDev *faces;
  const DftDev *dfts;
  const int *n_special;
  const int2 *pml_blocks, *special_blocks, *face_blocks, *dft_blocks;
  int n_pml_blocks, n_special_blocks, n_face_blocks, n_dft_blocks;
  int *const *d_bases;  // step counter of each active mesh
  int n_active;
};

// Blocks ahead of the running one whose PML data the batched kernel prefetches.
constexpr int kPmlBatchPrefetch = 1200;

// The batched PML kernel has the solo kernel's register budget: compiled
// for a different budget, the compiler fused some FP64 multiply-adds of the
// PML update differently, and in FP32 (where those values are rounded
// before they reach the links but reported unrounded) a few reported PML
// fields came out one rounding apart from the solo run.  With the same
// budget the two agree bit for bit.
template <typename T>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? TLM_PML_MIN_BLOCKS_FP32 : TLM_PML_MIN_BLOCKS)
    tlm_pml_batch_kernel(const BatchDev<T> b, int rel_step) {
  if (threadIdx.x == 0 && blockIdx.x + kPmlBatchPrefetch < b.n_pml_blocks) {
    const int2 f = b.pml_blocks[blockIdx.x + kPmlBatchPrefetch];  // (mesh, first cell)
    pml_prefetch_block<T>(b.meshes[f.x], b.pml[f.x], f.y, rel_step);
  }
  const int2 w = b.pml_blocks[blockIdx.x];
  const int s = w.y + threadIdx.x;
  const PmlList &pl = b.pml[w.x];
  if (s >= pl.n) return;
  pml_body<T>(b.meshes[w.x], pl, s, rel_step);
}

template <typename T, int MAXO>
__global__ void __launch_bounds__(128) tlm_special_batch_kernel(const BatchDev<T> b, int rel_step) {
  const int2 w = b.special_blocks[blockIdx.x];
  const int s = w.y + threadIdx.x;
  if (s >= b.n_special[w.x]) return;
  special_body<T, MAXO>(b.meshes[w.x], s, rel_step);
}

template <typename T>
__global__ void tlm_face_batch_kernel(const BatchDev<T> b, int rel_step) {
  const int2 w = b.face_blocks[blockIdx.x];
  const int f = w.y + threadIdx.x;
  const FaceDev &fd = b.faces[w.x];
  if (f >= fd.n_faces) return;
  face_body<T>(b.meshes[w.x], fd, f, rel_step);
}

template <typename T>
__global__ void tlm_dft_batch_kernel(const BatchDev<T> b, int rel_step) {
  const int2 w = b.dft_blocks[blockIdx.x];
  const int k = w.y + threadIdx.x;
  const DftDev &d = b.dfts[w.x];
  if (k >= d.n_entries) return;
  dft_body(d, b.meshes[w.x].d_base, k, rel_step);
}

__global__ void tlm_advance_batch(int *const *d_bases, int n_active, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_active) *d_bases[i] += n;
}

// TLM_set_small_to_zero (TLM_SOLVER/TLM_set_small_to_zero.F90:34-68), called
// before the excitation of every timestep that is a multiple of `every`
// (run_TLM.F90:236-238): incident pulses with |V| < small become 0.  Every
// slot of the buffer that step t reads holds exactly one cell's incident
// pulse (a neighbour's reflection, a face update written in place, or R times
// the cell's own reflection in a ghost slot), so the flush runs element-wise
// over that buffer; slots that no cell reads are padding.  The step number
// comes from the device counter, so the launch can sit in a replayed graph.
template <typename T>
__global__ void tlm_flush_small_kernel(const MeshDev<T> m, int rel_step, int every, double small) {
  const int t = *m.d_base + rel_step;
  if (t % every != 0) return;
  T *R = (t & 1) ? m.links0 : m.links1;  // written by step t-1
  const long long n4 = 12 * m.plane * (long long)sizeof(T) / 16;  // plane is a multiple of 4 elements
  uint4 *q = reinterpret_cast<uint4 *>(R);
  constexpr int E = 16 / sizeof(T);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
    uint4 w = q[i];
    T v[E];
    memcpy(v, &w, 16);
    bool hit = false;
#pragma unroll
    for (int e = 0; e < E; e++)
      if (fabs(double(v[e])) < small) { hit = hit || v[e] != T(0); v[e] = T(0); }
    if (hit) {
      memcpy(&w, v, 16);
      q[i] = w;
    }
  }
}

// Incident pulses of the next step in the reference layout V(12,nx,ny,nz):
// the same gather as the cell kernel, from the last written buffer.
template <typename T>
__global__ void tlm_gather_links(const MeshDev<T> m, int t_done, double *out) {
  const long long n = (long long)m.nx * m.ny * m.nz;
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= n) return;
  const int x = (int)(c % m.nx);
  const int y = (int)((c / m.nx) % m.ny);
  const int z = (int)(c / ((long long)m.nx * m.ny));
  const T *R = (t_done & 1) ? m.links1 : m.links0;
  const long long P = m.plane;
  const long long i = (long long)(z + 1) * m.PxPy + (long long)(y + 1) * m.Px + x;
  double *o = out + c * 12;
  o[Vy_xmin] = double(R[Vy_xmax * P + i - 1]);
  o[Vz_xmin] = double(R[Vz_xmax * P + i - 1]);
  o[Vy_xmax] = double(R[Vy_xmin * P + i + 1]);
  o[Vz_xmax] = double(R[Vz_xmin * P + i + 1]);
  o[Vx_ymin] = double(R[Vx_ymax * P + i - m.Px]);
  o[Vz_ymin] = double(R[Vz_ymax * P + i - m.Px]);
  o[Vx_ymax] = double(R[Vx_ymin * P + i + m.Px]);
  o[Vz_ymax] = double(R[Vz_ymin * P + i + m.Px]);
  o[Vx_zmin] = double(R[Vx_zmax * P + i - m.PxPy]);
  o[Vy_zmin] = double(R[Vy_zmax * P + i - m.PxPy]);
  o[Vx_zmax] = double(R[Vx_zmin * P + i + m.PxPy]);
  o[Vy_zmax] = double(R[Vy_zmin * P + i + m.PxPy]);
}

}  // namespace tlm
