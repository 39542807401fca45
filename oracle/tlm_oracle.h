/*
 * CPU oracle for the SCN-TLM time-stepping core -- TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C FP64 restatement of GGI_TLM's sequential time loop
 * (SRC/TLM_SOLVER/run_TLM.F90:191-295) on the reference's own data layout:
 * an array-of-structures link array V(1:12,0:nx+1,0:ny+1,1:nz)
 * (SRC/TLM_SOLVER/allocate_mesh.F90:120), a scatter pass over all cells
 * followed by a connect pass over all internal faces and an outer-boundary
 * pass, exactly in the reference's loop order and arithmetic order.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and only as the checker / CPU baseline.  The product
 * path (ggi_tlm_b200) never calls it.
 *
 * The problem tables are the arrays the reference's setup stage (L3) leaves
 * in its modules before run_TLM is called; the names follow the reference:
 *   cell_centre_update_code          SRC/TLM_MODULES/Mesh_Modules.F90:121
 *   cell_update_code_to_*            SRC/TLM_MODULES/Mesh_Modules.F90:139-150
 *   volume_material_list(:)          SRC/TLM_MODULES/TLM_material_modules.F90
 *   PML_parameters / PML_cell_data   SRC/TLM_MODULES/PML_module.F90:100-170
 *   excitation_functions(:)%value    SRC/EXCITATION/excitation.F90:155-559
 *   huygens_surface                  SRC/EXCITATION/huygens_surface.F90:247-715
 */
#ifndef TLM_ORACLE_H
#define TLM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_MAX_ORDER 8

typedef struct {
  /* mesh + solver parameters (set_TLM_solver_parameters.F90:94-96) */
  int32_t nx, ny, nz, n_timesteps;
  double dl, dt;
  double R[6]; /* R_xmin,R_xmax,R_ymin,R_ymax,R_zmin,R_zmax */

  /* cell update codes: nx*ny*nz entries in (cz,cy,cx) order, 0 or 1-based special index */
  const int32_t *cell_code;
  int32_t n_special;
  const int32_t *sp_material;   /* cell_update_code_to_material_data(:,1) */
  const int32_t *sp_pml;        /* cell_update_code_to_PML_data          */
  const int32_t *sp_excitation; /* cell_update_code_to_excitation_number */
  const int32_t *sp_output;     /* cell_update_code_to_output_number     */

  /* volume materials (1-based material numbers index these 0-based arrays) */
  int32_t n_materials;
  const int32_t *mat_type; /* 1 PEC, 2 PMC, 3 DISPERSIVE */
  const int32_t *mat_eps_exists, *mat_mu_exists;
  const int32_t *mat_eps_order, *mat_mu_order; /* Zfilter_response order */
  const double *mat_Ys_eps_f, *mat_Zs_mu_f, *mat_Ge, *mat_Rm;
  /* Zs_eps_Z / Zs_mu_Z coefficient rows, stride ORACLE_MAX_ORDER+1 */
  const double *mat_eps_a, *mat_eps_b, *mat_mu_a, *mat_mu_b;

  /* PML: 15 doubles per parameter row: ax,ay,az,exp_x,exp_y,exp_z,Csx,Csy,Csz,
     Csx2,Csy2,Csz2,Csy_sz,Csz_sx,Csx_sy (TLM_PML_volume_materials.F90:325-351) */
  int32_t n_pml_params;
  const double *pml_params;
  int32_t n_pml_cells;
  const int32_t *pml_cell_param; /* 1-based parameter index per PML cell */

  /* excitation function tables [n_fn][n_timesteps] */
  int32_t n_functions;
  const double *fn_value, *fn_value_face;

  /* cell-centre point excitations (excitation_points.F90:231-335) */
  int32_t n_exc_points;
  const int32_t *pt_cell; /* 1-based excitation cell number */
  const int32_t *pt_comp; /* 1..9 */
  const int32_t *pt_fn;   /* 1-based function */
  const int32_t *pt_type; /* 0 hard, 1 soft */
  int32_t n_exc_cells;

  /* special faces in connect order: 1-based cell (cx,cy,cz) on the + side of
     the face and the face normal axis 1..3; face_exc / face_out are 1-based
     excitation / output face numbers or 0 */
  int32_t n_faces;
  const int32_t *face_cx, *face_cy, *face_cz, *face_dir, *face_exc, *face_out;
  int32_t n_exc_faces, n_out_faces;

  /* Huygens surface (huygens_surface.F90:734-848) */
  int32_t hs_n;
  const int32_t *hs_face_exc; /* 1-based face excitation number per patch */
  const int32_t *hs_norm;     /* 3 ints per patch */
  const double *hs_offset;
  double hs_Ei[3], hs_Hi[3];
  double hs_offset_min, hs_c; /* c0/reduced_c_factor */
  int32_t hs_fn;              /* 1-based function */

  int32_t n_out_cells;

  /* frequency-domain output surfaces (frequency_output_surfaces.F90:297-421) */
  int32_t n_dft;
  const double *dft_freq;
  const int32_t *dft_comp;     /* 1..6 or 7..9 (Jx..Jz) */
  const int32_t *dft_face_ptr; /* CSR [n_dft+1] into dft_face_out / dft_face_side */
  const int32_t *dft_face_out; /* 1-based output face number */
  const int32_t *dft_face_side;/* 1..6 face code (face_xmin..face_zmax) */

  /* set_small_to_zero (read_small_to_zero.F90:55-59): every n_small_to_zero
     timesteps, |V| < small_to_zero_value -> 0; n_small_to_zero 0 = off */
  int32_t n_small_to_zero;
  double small_to_zero_value;

  /* PML_parameters(:)%sx,sy,sz (TLM_PML_volume_materials.F90:329-331), 3 per
     parameter row; needed by PML cells inside a volume material, else NULL */
  const double *pml_sigma;

  /* point sources on cell faces (EXCITATION/excitation_points.F90:286-323):
     1-based excitation face number, component 1..12, function, source type */
  int32_t n_face_points;
  const int32_t *fpt_face, *fpt_comp, *fpt_fn, *fpt_type;
  /* output points on cell faces (OUTPUT/output_points.F90:255-444): 1-based
     output face number, side 1 (min) / 2 (max), component 1..6 */
  int32_t n_face_probes;
  const int32_t *fprobe_face, *fprobe_side, *fprobe_comp;

  /* the Huygens surface is the outer boundary (huygens_surface%outer_surface_flag):
     its hs_n patches are boundary faces, 4 ints each in hs_cell (cx,cy,cz
     1-based, face code 1..6), and their sources enter in outer_boundary
     (TLM_SOLVER/outer_boundary.F90:133-318) instead of connect */
  int32_t hs_outer;
  const int32_t *hs_cell;

  /* far-field surfaces (OUTPUT/far_field_surfaces.F90:252-351), one entry
     per frequency: CSR list (ff_face_ptr[n_ff+1]) of 1-based output face
     numbers and face codes 1..6 of the face-list entry after the side flip */
  int32_t n_ff;
  const double *ff_freq;
  const int32_t *ff_face_ptr, *ff_face_out, *ff_face_code;

  /* surface materials on the special faces, connect_normal_to_x.F90:36-52
     (and the y, z analogues): per face 0 none, 1 PEC, 2 PMC, 4 free space
     (surface_material_type_*, TLM_MODULES/TLM_material_modules.F90:153-159);
     NULL: no surface materials */
  const int32_t *face_mat;

  /* thin layers on the special faces whose face_mat is 3 (surface material
     types DISPERSIVE and ANISOTROPIC_DISPERSIVE): per special face the
     signed thin-layer material number (1-based; positive: the layer is
     reversed, connect_normal_to_x.F90:14-19), and per material the fast
     parts f[3][4], the slow Z filters a, b [3][4][ORACLE_MAX_ORDER+1] and
     their orders [3][4] for the x, y, z polarisations and Z11, Z12, Z21,
     Z22 (TLM_surface_materials.F90:225-280) */
  const int32_t *face_smat;
  int32_t n_smat;
  const double *smat_f, *smat_a, *smat_b;
  const int32_t *smat_order;

  /* wrapping boundaries on x, y, z (0 or 1): wrap_outer_boundary after
     outer_boundary (TLM_SOLVER/wrap_outer_boundary.F90:101-273) */
  int32_t wrap[3];

  /* z-slab of a partitioned mesh (the reference's MPI build,
     general_mesh_subroutines.F90:868-972): slab[0] = 1 when a slab lies
     below (its top plane's Vx_zmax, Vy_zmax arrive in the ghost plane
     below this slab's first plane, and the z-faces between them are
     connected here), slab[1] = 1 when one lies above.  The outer boundary
     is not applied on such a side. */
  int32_t slab[2];

  /* output steps of each frequency output surface entry, [n_dft][3] =
     first, last, interval (get_output_flag, OUTPUT/output.F90:564-598);
     NULL: every step */
  const int32_t *dft_gate;

  /* the side of each face point source: 0 both (a point excitation,
     excitation_points.F90:286-323), 1 or 2 that side alone (a one-sided
     excitation surface, excitation_surfaces.F90:236-262); NULL: all 0 */
  const int32_t *fpt_side;

  /* the factor on the function's value of each face point source: a mode
     excitation's mode field, halved on both sides (Mode_excitation,
     mode_excitation.F90:393-411); NULL: all 1 */
  const double *fpt_scale;
} tlm_oracle_problem;

typedef struct tlm_oracle_state tlm_oracle_state;

tlm_oracle_state *tlm_oracle_create(const tlm_oracle_problem *p);
void tlm_oracle_destroy(tlm_oracle_state *s);
/* run timesteps first..first+n-1 (1-based, reference numbering); cell_out
   receives n x n_out_cells x 6 doubles (cell_output_field after each scatter) */
int tlm_oracle_run(tlm_oracle_state *s, int32_t first_step, int32_t n_steps, double *cell_out);
/* DFT accumulators: per surface, per face, (re,im) */
int tlm_oracle_get_dft(tlm_oracle_state *s, double *out);
/* far-field accumulators per surface face: J(3), M(3) as (re, im) pairs */
int tlm_oracle_get_far_field(tlm_oracle_state *s, double *out);
/* face output point values of every completed timestep: [timestep][n_face_probes] */
int tlm_oracle_get_face_probes(tlm_oracle_state *s, double *out);
/* link array dump in the reference layout V(12, nx, ny, nz) interior only */
int tlm_oracle_get_links(tlm_oracle_state *s, double *out);
/* host threads for the scatter and connect passes (z-planes shared among
   them, as the reference's MPI build shares z-slabs among ranks); the
   arithmetic of every cell and face is unchanged, so the results are the
   same for any count (at most 256).  Returns the count in use. */
int tlm_oracle_set_threads(tlm_oracle_state *s, int32_t threads);
/* one timestep in the two halves a partitioned run exchanges data between
   (run_TLM.F90:242-291): half 1 = excitation, scatter, cell_output (then
   TLM_parallel_pass_data_1); half 2 = connect, face outputs, outer boundary,
   wrapping (then TLM_parallel_pass_data_2).  tlm_oracle_run does both. */
int tlm_oracle_half_step(tlm_oracle_state *s, int32_t timestep, int32_t half, double *cell_out);
/* the two ports of a z-plane the passes carry, as [2][ny][nx] (Vx_zmax,
   Vy_zmax), TLM_parallel_pass_data.F90:38-279: plane 0 = the ghost plane
   below the slab, plane 1 = the slab's top plane */
int tlm_oracle_get_zplane(tlm_oracle_state *s, int32_t plane, double *out);
int tlm_oracle_set_zplane(tlm_oracle_state *s, int32_t plane, const double *in);

#ifdef __cplusplus
}
#endif
#endif
