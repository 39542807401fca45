/*
 * tlm_gpu.h -- C-ABI of the B200 (sm_100a) SCN-TLM time-stepping core.
 *
 * Drop-in boundary for GGI_TLM's time loop: the unchanged Fortran driver
 * (SRC/GGI_TLM.F90) runs all of its setup (input parsing, .mesh reading,
 * materials, PML, excitation and output set-up) and then, in place of
 * `CALL run_TLM()` (SRC/GGI_TLM.F90:157), hands the module arrays below to
 * this library and advances the mesh on the GPU.  The pattern follows the
 * reference's only existing Fortran->C binding, MODULE ngspice_F90
 * (SRC/NGSPICE_LINK/run_ngspice_TLM.F90:40-110): ISO_C_BINDING interfaces,
 * scalars and arrays by reference, an integer return code.
 *
 * Conventions
 *  - All pointers are caller-owned host memory.  The library copies what it
 *    needs at set-time and never keeps a caller pointer.
 *  - Indices inside the arrays are the reference's 1-based numbers
 *    (special cell codes, material numbers, PML cell numbers, excitation and
 *    output numbers), so the Fortran arrays pass through unchanged.
 *  - Every entry point returns TLM_OK (0) or a negative TLM_E_* code;
 *    tlm_gpu_last_error() returns the message of the last failure on the
 *    calling thread.  The Fortran shim maps a non-zero code to
 *    `write(*,*) msg; STOP 1`, the reference's own convention
 *    (set_update_codes.F90:316, scatter.F90:561-567).
 *  - One host thread per handle.  The library launches on its own CUDA
 *    stream unless tlm_gpu_set_stream() gives it one.
 *  - Features outside the GPU path (cables, Ngspice, diode/switch/SPICE-port
 *    surface materials, periodic boundaries, mode stirring, PML cells inside
 *    dispersive materials) are rejected with TLM_E_UNSUPPORTED at set-time.
 *    The MPI build's z-slabs map to one mesh per slab with the halo calls
 *    (tlm_gpu_halo_get / tlm_gpu_halo_put).
 */
#ifndef TLM_GPU_H
#define TLM_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TLM_OK 0
#define TLM_E_BADARG (-1)
#define TLM_E_UNSUPPORTED (-2)
#define TLM_E_OOM (-3)
#define TLM_E_CUDA (-4)
#define TLM_E_STATE (-5)
#define TLM_E_TIMEOUT (-6)

#define TLM_PRECISION_FP32 32 /* FP32 links + FP32 scatter; FP64 filters, sources, DFT */
#define TLM_PRECISION_FP64 64 /* plain FP64 everywhere (parity path) */

#define TLM_MAX_FILTER_ORDER 8

/* Mesh and solver parameters: nx,ny,nz (TLM_general), dl, dt
   (set_TLM_solver_parameters.F90:94), n_timesteps (:96) and the outer
   boundary reflection coefficients R_xmin..R_zmax (outer_boundary.F90). */
typedef struct tlm_gpu_mesh_desc {
  int32_t nx, ny, nz;
  int32_t n_timesteps;
  double dl, dt;
  double R[6];
  int32_t precision; /* TLM_PRECISION_FP32 or TLM_PRECISION_FP64 */
  int32_t device;    /* CUDA device ordinal */
} tlm_gpu_mesh_desc;

/* Allocate device state for one mesh; replaces allocate_mesh
   (SRC/TLM_SOLVER/allocate_mesh.F90:106-134).  Links start at zero. */
int tlm_gpu_create(const tlm_gpu_mesh_desc *desc, int64_t *handle);

/* Cell classification: cell_centre_update_code(1:nx*ny*nz) in (cz,cy,cx)
   order and the lookup tables cell_update_code_to_material_data(:,1),
   cell_update_code_to_PML_data, cell_update_code_to_excitation_number,
   cell_update_code_to_output_number (SRC/TLM_MODULES/Mesh_Modules.F90:121-150,
   built by set_cell_update_codes, SRC/TLM_SOLVER/set_update_codes.F90:38-363).
   Cable numbers must be zero. */
int tlm_gpu_set_cells(int64_t handle, const int32_t *cell_centre_update_code, int32_t n_special,
                      const int32_t *sp_material, const int32_t *sp_pml, const int32_t *sp_excitation,
                      const int32_t *sp_output);

/* Volume materials: volume_material_list(1:n) after
   calculate_volume_material_filter_coefficients
   (SRC/MATERIALS/TLM_volume_materials.F90:190-385): type (1 PEC, 2 PMC,
   3 DISPERSIVE), filter existence flags, Zfilter_response orders, Ys_eps_f,
   Zs_mu_f, Ge, Rm and the Zs_eps_Z / Zs_mu_Z coefficient rows a(0:order),
   b(0:order) laid out with row stride `coeff_stride` (>= order+1). */
int tlm_gpu_set_materials(int64_t handle, int32_t n_materials, const int32_t *type, const int32_t *eps_exists,
                          const int32_t *mu_exists, const int32_t *eps_order, const int32_t *mu_order,
                          const double *Ys_eps_f, const double *Zs_mu_f, const double *Ge, const double *Rm,
                          const double *eps_a, const double *eps_b, const double *mu_a, const double *mu_b,
                          int32_t coeff_stride);

/* PML: PML_parameters(1:n_params) as 15 doubles per row in the order
   ax,ay,az,exp_x,exp_y,exp_z,Csx,Csy,Csz,Csx2,Csy2,Csz2,Csy_sz,Csz_sx,Csx_sy
   (SRC/TLM_MODULES/PML_module.F90:100-113, filled at
   SRC/MATERIALS/TLM_PML_volume_materials.F90:325-351) and
   PML_cell_data(1:n_pml_cells)%PML_parameter_array_pos. */
int tlm_gpu_set_pml(int64_t handle, int32_t n_params, const double *params, int32_t n_pml_cells,
                    const int32_t *pml_cell_param);

/* PML_parameters(1:n_params)%sx,sy,sz: the layer conductivities divided by
   eps0 (SRC/MATERIALS/TLM_PML_volume_materials.F90:321-331), 3 doubles per
   row.  Required (after tlm_gpu_set_pml) when a PML cell lies inside a
   volume material: those cells take the PML-material update
   (SRC/TLM_SOLVER/scatter_PML_material.F90:22-534), which rebuilds its
   recursion coefficients from them.  The caller keeps the reference's
   precondition (SRC/TLM_SOLVER/set_update_codes.F90:290-331): such a
   material has eps_r and mu_r of S-domain order 0. */
int tlm_gpu_set_pml_sigma(int64_t handle, int32_t n_params, const double *sigma);

/* Excitation: excitation_functions(1:n_fn)%value(1:n_steps) and
   %value_face(1:n_steps) (SRC/EXCITATION/excitation.F90:155-559), and the
   cell-centre point excitations (excitation cell number, field component
   1..9, function number, source type 0 hard / 1 soft) of
   SRC/EXCITATION/excitation_points.F90:231-335. */
int tlm_gpu_set_excitation(int64_t handle, int32_t n_functions, int32_t n_steps, const double *value,
                           const double *value_face, int32_t n_points, const int32_t *pt_cell,
                           const int32_t *pt_comp, const int32_t *pt_fn, const int32_t *pt_type,
                           int32_t n_exc_cells);

/* Special faces, the non-zero entries of face_update_code compacted in
   connect order (SRC/TLM_SOLVER/connect.F90:180-214): 1-based cell
   (cx,cy,cz) on the + side of the face, normal axis 1..3, 1-based face
   excitation number (or 0) and face output number (or 0).  Surface
   materials are not part of the GPU path. */
int tlm_gpu_set_faces(int64_t handle, int32_t n_faces, const int32_t *cx, const int32_t *cy, const int32_t *cz,
                      const int32_t *dir, const int32_t *exc, const int32_t *out, int32_t n_exc_faces,
                      int32_t n_out_faces);

/* Surface materials on the special faces, in set_faces order
   (face_update_code_to_material_data, connect_normal_to_x.F90:20-52 and the
   y, z analogues): 0 none, 1 PEC (surface_material_type_PEC: each side
   reflects its own pulse with -1), 2 PMC (+1), 3 a dispersive thin layer
   (tlm_gpu_set_thin_layers, tlm_gpu_set_face_thin_layers), 4 free space
   (the plain connect).  Other surface material types (switches, diodes,
   spice ports) are rejected with TLM_E_UNSUPPORTED at the first run.
   Without this call no special face carries a material. */
int tlm_gpu_set_face_materials(int64_t handle, int32_t n_faces, const int32_t *type);

/* Dispersive thin layers (surface material types DISPERSIVE and
   ANISOTROPIC_DISPERSIVE; replaces calculate_surface_material_filter_
   coefficients, MATERIALS/TLM_surface_materials.F90:225-280, whose results
   the Fortran driver passes here).  n materials; for material i,
   polarisation p (x, y, z) and filter k (Z11, Z12, Z21, Z22), entry
   e = (i*3 + p)*4 + k: the fast part f[e], the slow Z filter's
   coefficients a[e*stride .. e*stride+order[e]] and b[...] (b(0) != 0).
   Orders above 8 and impedance matrices that surface_material_update
   could not solve are rejected. */
int tlm_gpu_set_thin_layers(int64_t handle, int32_t n, const double *f, const double *a, const double *b,
                            const int32_t *order, int32_t stride);

/* Per special face (tlm_gpu_set_faces order) the signed thin-layer
   material, face_update_code_to_material_data(:,1) of a thin-layer face:
   0 none, +m material m with the layer reversed, -m not reversed
   (connect_normal_to_x.F90:14-19).  A face with a thin layer has surface
   material type 3 in tlm_gpu_set_face_materials. */
int tlm_gpu_set_face_thin_layers(int64_t handle, int32_t n, const int32_t *material);

/* Wrapping boundaries (Wrapping_boundary_conditions packet, wrap_x/y/z;
   TLM_SOLVER/wrap_outer_boundary.F90:101-273): on a wrapped axis the two
   outer faces are joined, each boundary port receiving R times the
   reflected pulse of the cell at the other end (the reference swaps the
   two ends' ports after outer_boundary).  Flags 0 or 1.  Not with an
   outer-boundary Huygens surface (TLM_E_UNSUPPORTED at the first run). */
int tlm_gpu_set_wrap(int64_t handle, int32_t wrap_x, int32_t wrap_y, int32_t wrap_z);

/* Huygens surface (SRC/EXCITATION/huygens_surface.F90:247-848): per patch
   the face excitation number, normal (3 ints) and offset; the incident
   field vectors Ei, Hi; offset_min, the wave speed c0/reduced_c and the
   excitation function number. */
int tlm_gpu_set_huygens(int64_t handle, int32_t n_patches, const int32_t *face_exc, const int32_t *norm,
                        const double *offset, const double *Ei, const double *Hi, double offset_min, double c,
                        int32_t function);

/* The Huygens surface on the outer boundary of the mesh (surface number 0
   of the Huygens_surface packet; SRC/EXCITATION/huygens_surface.F90:508-612):
   n boundary faces, 4 ints each (cx, cy, cz 1-based, face code 1..6 with
   the outward normal of the mesh), their offsets K.r, the field vectors,
   offset_min, c0/reduced_c and the excitation function.  Their J, M are
   added to the boundary ports after the R reflection
   (SRC/TLM_SOLVER/outer_boundary.F90:133-318).  Use it in place of
   tlm_gpu_set_huygens: the reference has one Huygens surface. */
int tlm_gpu_set_outer_huygens(int64_t handle, int32_t n_faces, const int32_t *cell_face, const double *offset,
                              const double *Ei, const double *Hi, double offset_min, double c, int32_t function);

/* Point sources on cell faces (SRC/EXCITATION/excitation_points.F90:
   135-211 numbering, :286-323 per step): 1-based excitation face number of
   the face (the min face of the cell on its + side, as in set_faces),
   component 1..12 (Ex..Hz, Jx..Jz, Mx..Mz), excitation function, source type
   (0 hard, 1 soft).  value_face(timestep) of the function is added on both
   sides of the face, and the type of the E/H component set there; connect
   then applies them (SRC/TLM_SOLVER/connect_normal_to_x.F90:287-307 and the
   y, z analogues).  Every excitation face needs a Huygens patch or a point. */
int tlm_gpu_set_face_excitation(int64_t handle, int32_t n_points, const int32_t *face_exc, const int32_t *component,
                                const int32_t *function, const int32_t *source_type);

/* Excitation surfaces (SRC/EXCITATION/excitation_surfaces.F90:218-275) as
   face sources, listed after the point sources: per entry of
   tlm_gpu_set_face_excitation 0 (both sides, a point source or a surface
   with side 0) or the one side, 1 (min) or 2 (max), that receives the
   value; a source type set on side 2 alone does not reach connect, which
   reads side 1's types on both sides.  Optional: without it every entry
   reaches both sides.  Replaces Surface_excitation's face loop. */
int tlm_gpu_set_face_excitation_side(int64_t handle, int32_t n_points, const int32_t *side);

/* Mode excitations (SRC/EXCITATION/mode_excitation.F90:330-420) as face
   sources listed last: per entry of tlm_gpu_set_face_excitation the factor
   on the function's value, the face's mode field on one side, or half of it
   on both sides (side 0 of the packet).  Optional: without it every factor
   is 1.  Replaces Mode_excitation's face loop. */
int tlm_gpu_set_face_excitation_scale(int64_t handle, int32_t n_points, const double *scale);

/* Output points on cell faces (SRC/OUTPUT/output_points.F90:255-444):
   1-based output face number, side (1 = the min-side field, face_xmin/ymin/
   zmin; 2 = the max side) and component 1..6 of face_output_field after
   connect, recorded every step. */
int tlm_gpu_set_face_outputs(int64_t handle, int32_t n_points, const int32_t *face_out, const int32_t *side,
                             const int32_t *component);

/* Number of output cells; cell_output_field(1:n,1:6) is recorded every
   step (SRC/TLM_SOLVER/scatter.F90:465-480, scatter_PML.F90 STAGE 12). */
int tlm_gpu_set_outputs(int64_t handle, int32_t n_out_cells);

/* Which output cells keep a time series: keep[i] = 1 for output cell i+1
   when its cell_output_field rows are read back step by step (the output
   points, SRC/OUTPUT/output_points.F90:463-612), 0 when only volume outputs
   read it.  Without this call every output cell keeps one.  No counterpart
   in the reference, which writes output points to file every step and
   keeps no history. */
int tlm_gpu_set_output_series(int64_t handle, int32_t n_out_cells, const int32_t *keep);

/* Frequency output volumes (SRC/OUTPUT/frequency_output_volumes.F90:35-390),
   one entry per volume and frequency as frequency_output_volume(:):
   frequency, field component 1..6 (Ex..Hz), first_timestep, last_timestep
   and timestep_interval (SRC/OUTPUT/output.F90:564-598), and a CSR list
   (cell_ptr[n_volumes+1]) of the 1-based output cell numbers of the
   volume's cells (cell_output_field_number_list).  On each output step
   value += cell_output_field(cell, component) exp(-j 2 pi f (timestep-1) dt). */
int tlm_gpu_set_volume_dft(int64_t handle, int32_t n_volumes, const double *frequency, const int32_t *component,
                           const int32_t *first_step, const int32_t *last_step, const int32_t *interval,
                           const int32_t *cell_ptr, const int32_t *cell_out);

/* Frequency output volume values per volume cell in set_volume_dft order,
   (re, im) pairs: frequency_output_volume(:)%value(:). */
int tlm_gpu_fetch_volume_dft(int64_t handle, double *out);

/* Time-domain output volumes: kind 0 = output_volumes(:) (each cell's
   field, SRC/OUTPUT/output_volumes.F90), 1 = output_volume_averages(:)
   (the mean over the cells, output_volume_averages.F90), 2 =
   output_volume_peak(:) (the largest |field|, output_volume_peak.F90);
   field component 1..6, first_timestep, last_timestep, timestep_interval
   and a CSR list (cell_ptr[n+1]) of the 1-based output cell numbers
   (cell_output_field_number_list).  Averages and peaks below 1e-30 in
   magnitude are recorded as 0, as the reference writes them. */
int tlm_gpu_set_output_volumes(int64_t handle, int32_t n_volumes, const int32_t *kind, const int32_t *component,
                               const int32_t *first_step, const int32_t *last_step, const int32_t *interval,
                               const int32_t *cell_ptr, const int32_t *cell_out);

/* Output volume values, volume after volume: kind 0 [n_output_steps][n_cells],
   kinds 1 and 2 [n_output_steps], n_output_steps = the steps
   first..min(last, n_timesteps) every interval; rows of steps not run yet
   are zero. */
int tlm_gpu_fetch_output_volumes(int64_t handle, double *out);

/* SAR volumes (SRC/OUTPUT/SAR_volumes.F90:36-330), one entry per volume
   and frequency as SAR_volume_list(:): frequency and a CSR list
   (cell_ptr[n+1]) of the 1-based output cell numbers of the volume's
   cells.  Every step each cell accumulates Ex, Ey, Ez +=
   exp(-j 2 pi f (timestep-1) dt) * field * dt; write_SAR_volumes turns
   them into SAR on the host. */
int tlm_gpu_set_sar_volumes(int64_t handle, int32_t n_volumes, const double *frequency, const int32_t *cell_ptr,
                            const int32_t *cell_out);

/* SAR volume accumulators per cell in set_sar_volumes order: Ex, Ey, Ez as
   (re, im) pairs, 6 doubles per cell (SAR_volume_list(:)%Ex(:), %Ey, %Ez). */
int tlm_gpu_fetch_sar_volumes(int64_t handle, double *out);

/* Time-domain output surfaces (SRC/OUTPUT/output_surfaces.F90:42-760), as
   output_surfaces(:): field component (1..6 Ex..Hz, 7..9 Jx..Jz = n x H,
   13 |E|, 14 |H|, 15 |J|), first_timestep, last_timestep, timestep_interval,
   output_average_of_both_sides (0/1), and a CSR list (face_ptr[n+1]) of the
   surface's faces: output face number and face code 1..6 after the side
   flip (output_on_outward_normal).  On each output step every face's
   value (face_output_surfaces, :601-760) is recorded. */
int tlm_gpu_set_output_surfaces(int64_t handle, int32_t n_surfaces, const int32_t *component,
                                const int32_t *first_step, const int32_t *last_step, const int32_t *interval,
                                const int32_t *both_sides, const int32_t *face_ptr, const int32_t *face_out,
                                const int32_t *face_code);

/* Output surface values, surface after surface, each [n_output_steps][n_faces]
   doubles, n_output_steps = the steps first..min(last, n_timesteps) every
   interval; rows of steps not run yet are zero. */
int tlm_gpu_fetch_output_surfaces(int64_t handle, double *out);

/* The RCS surface (SRC/OUTPUT/RCS_surfaces.F90:159-560, rcs_surface):
   theta and phi in radians, n_rcs_points_per_cell, n_far_field_points and
   far_field_point_offset as initialise_rcs_surfaces sets them, and the
   surface's faces: output face number, face code 1..6 after the side flip
   and K.x of the face point (get_cell_point_coordinate).  Every step each
   face adds its far-field contribution to Etheta/Ephi/Htheta/Hphi at point
   INT(n_rcs_points_per_cell ((time c0) - K.x) / dl) - far_field_point_offset,
   time = (timestep-1) dt + dt/2; points outside 1..n_far_field_points are
   dropped, as the reference drops them after its warning. */
int tlm_gpu_set_rcs(int64_t handle, double theta, double phi, int32_t points_per_cell, int32_t n_points,
                    int32_t point_offset, int32_t n_faces, const int32_t *face_out, const int32_t *face_code,
                    const double *face_dist);

/* RCS far-field arrays: Etheta, Ephi, Htheta, Hphi, each n_points doubles. */
int tlm_gpu_fetch_rcs(int64_t handle, double *out);

/* Frequency-domain power surfaces
   (SRC/OUTPUT/frequency_domain_power_surfaces.F90:35-420), one entry per
   surface and frequency (fmin + (k-1) fstep): frequency and a CSR list
   (face_ptr[n+1]) of output face numbers and face codes 1..6.  Every step
   each face accumulates E1, E2, H1, H2 (the tangential fields on its side)
   times exp(-j 2 pi f t) at the face-output time. */
int tlm_gpu_set_power_surfaces(int64_t handle, int32_t n, const double *frequency, const int32_t *face_ptr,
                               const int32_t *face_out, const int32_t *face_code);

/* Power surface accumulators per face in set order: E1, E2, H1, H2 as
   (re, im) pairs, 8 doubles per face. */
int tlm_gpu_fetch_power_surfaces(int64_t handle, double *out);

/* Mode outputs (SRC/OUTPUT/output_modes.F90:35-620), as output_mode_list(:):
   field component 1..6 and a CSR list (face_ptr[n+1]) of the mode samples:
   output face number, face code 1..6 and mode_field.  Every step each
   mode's value is the sum of face_output_field(side, component) *
   mode_field over its faces, 0 below 1e-30 in magnitude. */
int tlm_gpu_set_mode_outputs(int64_t handle, int32_t n_modes, const int32_t *component, const int32_t *face_ptr,
                             const int32_t *face_out, const int32_t *face_code, const double *mode_field);

/* Mode output values of steps first..first+n-1: out[n][n_modes]. */
int tlm_gpu_fetch_mode_outputs(int64_t handle, int32_t first_step, int32_t n_steps, double *out);

/* Frequency-domain output surfaces (one entry per frequency, as
   frequency_output_surface(:) in SRC/OUTPUT/frequency_output_surfaces.F90:
   297-421): frequency, field component (1..6 E/H, 7..9 J=nxH), and a CSR
   list (face_ptr[n_surfaces+1]) of output face numbers and face codes
   (1..6 = face_xmin,ymin,zmin,xmax,ymax,zmax). */
int tlm_gpu_set_dft(int64_t handle, int32_t n_surfaces, const double *frequency, const int32_t *component,
                    const int32_t *face_ptr, const int32_t *face_out, const int32_t *face_code);

/* Output steps of each frequency-domain output surface entry (call after
   tlm_gpu_set_dft, same count): timesteps first..last every interval
   contribute (get_output_flag, SRC/OUTPUT/output.F90:564-598, as
   face_output_frequency_output_surfaces applies it,
   frequency_output_surfaces.F90:336-342).  Without this call every step
   contributes. */
int tlm_gpu_set_dft_gate(int64_t handle, int32_t n_surfaces, const int32_t *first_timestep,
                         const int32_t *last_timestep, const int32_t *timestep_interval);

/* set_small_to_zero packet (SRC/PROCESS_INPUT_FILE/read_small_to_zero.F90:
   55-59): before the excitation of every timestep that is a multiple of
   n_small_to_zero, incident link pulses with |V| < small_to_zero_value
   become 0 (SRC/TLM_SOLVER/TLM_set_small_to_zero.F90:34-68, called at
   run_TLM.F90:236-238).  n_small_to_zero = 0 switches it off (the default). */
int tlm_gpu_set_small_to_zero(int64_t handle, int32_t n_small_to_zero, double small_to_zero_value);

/* Far-field surfaces (SRC/OUTPUT/far_field_surfaces.F90:36-351), one entry
   per frequency as far_field_surface(:): frequency and a CSR list
   (face_ptr[n_surfaces+1]) of output face numbers and face codes 1..6 of
   the surface's faces after the side flip.  Every step each face
   accumulates J += exp(-j 2 pi f t) dt (n x H) and M -= exp(-j 2 pi f t) dt
   (n x E) on its side of face_output_field, n = +1 on a min face, -1 on a
   max face. */
int tlm_gpu_set_far_field(int64_t handle, int32_t n_surfaces, const double *frequency, const int32_t *face_ptr,
                          const int32_t *face_out, const int32_t *face_code);

/* Far-field accumulators per surface face in set_far_field order: Jx, Jy,
   Jz, Mx, My, Mz as (re, im) pairs, 12 doubles per face. */
int tlm_gpu_fetch_far_field(int64_t handle, double *out);

/* Build the handle's device state now (allocations, table uploads, masks)
   instead of at its first run; a serving loop calls it for a new request
   while other solves are running.  No counterpart in the reference, which
   sets up once before run_TLM. */
int tlm_gpu_prepare(int64_t handle);

/* Advance timesteps first_step..first_step+n_steps-1 (1-based, run_TLM
   numbering, SRC/TLM_SOLVER/run_TLM.F90:191-295).  Steps must be
   contiguous across calls.  Asynchronous on the library stream. */
int tlm_gpu_run(int64_t handle, int32_t first_step, int32_t n_steps);

/* Block until all work of the handle has finished. */
int tlm_gpu_synchronize(int64_t handle);

/* cell_output_field snapshots of steps first..first+n-1 of the output
   cells that keep a time series (all of them unless set_output_series
   says otherwise), in output-number order: out[n][n_kept][6] doubles. */
int tlm_gpu_fetch_cell_output(int64_t handle, int32_t first_step, int32_t n_steps, double *out);

/* Face output point values of steps first..first+n-1: out[n][n_points]
   (the time of step k is (k-1)*dt + dt/2, output_points.F90:441). */
int tlm_gpu_fetch_face_output(int64_t handle, int32_t first_step, int32_t n_steps, double *out);

/* DFT accumulators (re, im) per surface face in set_dft order. */
int tlm_gpu_fetch_dft(int64_t handle, double *out);

/* Incident link voltages of the next step in the reference layout
   V(1:12,1:nx,1:ny,1:nz) (port fastest), i.e. the content of the
   reference's V array after outer_boundary. */
int tlm_gpu_fetch_links(int64_t handle, double *out);

/* Allocation-free variant of tlm_gpu_fetch_links.  It has no counterpart in
   the reference.  It exists for callers that cannot call cudaMalloc: code
   that must not grow device memory it does not own (a host framework with a
   fixed device budget or pool), or that must not trigger the implicit device
   synchronisation of cudaMalloc/cudaFree while other GPU work is in flight.
   The gather runs into a fixed scratch array inside the library (8 MiB per
   device that loads the library, kept until the process exits), so the mesh
   may have at most 87381 cells (nx*ny*nz*12 <= 2^20 doubles); larger meshes
   are rejected with TLM_E_BADARG.  The mesh must already have device state
   (built by tlm_gpu_prepare, tlm_gpu_run or tlm_gpu_batch_create; before
   any run it returns the initial, all-zero links).  A mesh that belongs to
   a batch is read after the batch's queued steps finish.  The first call on a device looks up the
   scratch address (cudaGetSymbolAddress) and should come before any stream
   capture.  All calls share the one scratch array, which keeps the last
   call's contents: calls that overlap on the GPU (other host threads, other
   handles) race on it. */
int tlm_gpu_fetch_links_noalloc(int64_t handle, double *out);

/* z-slab halo exchange of a mesh that is one slab of a partitioned mesh
   (replaces TLM_SOLVER/TLM_parallel_pass_data.F90:38-279, the MPI passes
   between z-slab ranks; slabs as MESH/general_mesh_subroutines.F90:868-972
   assigns them).  Between two timesteps, the slab below needs this slab's
   first-plane Vx_zmin, Vy_zmin pulses in its ghost plane above, and the slab
   above needs its last-plane Vx_zmax, Vy_zmax pulses in its ghost plane
   below.  One side is two ports of one padded z-plane, *bytes bytes
   (tlm_gpu_halo_bytes; slabs of one mesh have equal sizes).
     tlm_gpu_halo_get side 0: this slab's first plane (Vx_zmin, Vy_zmin),
                      side 1: its last plane (Vx_zmax, Vy_zmax);
     tlm_gpu_halo_put side 0: the ghost plane below (Vx_zmax, Vy_zmax),
                      side 1: the ghost plane above (Vx_zmin, Vy_zmin).
   Both act on the pulses the last completed step reflected (the ones the
   next step reads), with device-to-device copies on the mesh's stream
   between `dev` (device memory of this mesh's device, or peer memory the
   device can reach) and the link planes, and return once the copies are
   done.  The mesh's outer boundary on a slab side is overwritten by the
   put, so its R there does not matter. */
int tlm_gpu_halo_bytes(int64_t handle, int64_t *bytes);
int tlm_gpu_halo_get(int64_t handle, int32_t side, void *dev);
int tlm_gpu_halo_put(int64_t handle, int32_t side, const void *dev);

/* Test hook for the bounded waits (no counterpart in the reference): adds
   `bytes` (a multiple of 16, at most 4096; 0 = normal operation) to the byte
   count that every bulk-copy wait of the mesh's TMA cell kernel expects.
   The copies all complete, but the waits cannot, so each runs out after its
   2 s limit, the kernel records TLM_E_TIMEOUT and returns, and the next
   tlm_gpu_synchronize (or tlm_gpu_batch_synchronize) reports it.  The mesh's
   results are then invalid; the device context stays usable. */
int tlm_gpu_set_test_wait_pad(int64_t handle, int32_t bytes);

/* Use a caller CUDA stream (cudaStream_t passed as void*; NULL = own). */
int tlm_gpu_set_stream(int64_t handle, void *stream);

/* Kernel timing mode: when enabled, tlm_gpu_run launches step by step
   (no graph replay) and brackets every fused cell kernel with CUDA events on
   the launch stream, so tlm_gpu_last_run_time can report the summed cell
   kernel time of the run. */
int tlm_gpu_set_timing(int64_t handle, int32_t enable);

/* Tuning: select the configuration of the bulk (free-space) cell kernel,
   0 = register-pipelined kernel, 1..n-1 = TMA-staged persistent kernel
   with different tile sizes and shared-memory ring depths.  Numerics are
   identical for every variant; the autotuner picks the fastest. */
int tlm_gpu_set_variant(int64_t handle, int32_t variant);
int tlm_gpu_num_variants(int32_t *n_variants);

/* Device time of the last tlm_gpu_run (CUDA events on the launch stream):
   whole run, and the summed duration of the fused cell kernel alone. */
int tlm_gpu_last_run_time(int64_t handle, float *ms_total, float *ms_cell_kernel);

/* Device memory held by the handle, bytes. */
int tlm_gpu_memory_bytes(int64_t handle, int64_t *bytes);

/* Number of kernel launches issued by the last tlm_gpu_run. */
int tlm_gpu_last_run_launches(int64_t handle, int64_t *launches);

int tlm_gpu_destroy(int64_t handle);

/* Batches (no counterpart in the reference, which runs one mesh per
   process): advance many meshes of one precision together.  Every batch
   step is one persistent TMA-staged launch over the concatenated tile lists
   of all active meshes plus one launch each for their PML cells, other
   special cells, special faces and DFT entries, captured once as a CUDA
   graph and replayed.  Each mesh runs until its own n_timesteps; a mesh that
   finishes drops out and the work lists are rebuilt.  Results are read per
   mesh with the tlm_gpu_fetch_* calls (after tlm_gpu_batch_synchronize).
   A mesh may belong to one batch at a time and must not be run on its own
   while it does. */
int tlm_gpu_batch_create(const int64_t *handles, int32_t n_meshes, int64_t *batch);
int tlm_gpu_batch_set_variant(int64_t batch, int32_t variant);
/* Replace the meshes of a batch (same precision and device; a mesh may stay,
   leave or join).  The batch first waits for its queued steps; meshes that
   leave can then be run alone, read or destroyed, and the work lists are
   rebuilt at the next tlm_gpu_batch_run.  The batch keeps its stream, graph
   resources and device buffers, so a serving loop changes membership
   without destroying and creating batches. */
int tlm_gpu_batch_set_members(int64_t batch, const int64_t *handles, int32_t n_meshes);
/* Advance every unfinished mesh by up to n_steps steps (asynchronous). */
int tlm_gpu_batch_run(int64_t batch, int32_t n_steps);
int tlm_gpu_batch_synchronize(int64_t batch);
/* Device time, cell updates and kernel launches of the last batch run. */
int tlm_gpu_batch_last_run(int64_t batch, float *ms, int64_t *cell_updates, int64_t *launches);
int tlm_gpu_batch_destroy(int64_t batch);

/* Message of the last failure on this thread (NUL-terminated, truncated
   to len-1 characters). */
/* Device-memory cache of the library (no counterpart in the reference,
   whose arrays are allocated once per run): buffers of destroyed meshes and
   batches are kept per device, up to TLM_POOL_CACHE_BYTES (default 16 GiB),
   and reused by later meshes, so creating and destroying meshes in a
   serving loop does not call cudaMalloc/cudaFree each time.
   tlm_gpu_pool_release returns every cached block to the driver;
   tlm_gpu_pool_cached_bytes reports how much is cached. */
int tlm_gpu_pool_release(void);
int tlm_gpu_pool_cached_bytes(int64_t *bytes);

int tlm_gpu_last_error(char *buf, int32_t len);

#ifdef __cplusplus
}
#endif
#endif /* TLM_GPU_H */
