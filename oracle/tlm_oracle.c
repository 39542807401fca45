/*
 * CPU oracle for the SCN-TLM time-stepping core -- TEST INFRASTRUCTURE ONLY.
 * See tlm_oracle.h for the data contract.  Every routine cites the reference
 * routine it restates; loop order and arithmetic order follow the reference
 * so that the oracle reproduces GGI_TLM_SEQ's probe series to rounding.
 */
#include "tlm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

/* SRC/CONSTANTS/constants.F90:27-39 */
static const double Z0 = 376.73031346177;
#define Y0 (1.0 / Z0)

/* port numbering, SRC/TLM_MODULES/Mesh_Modules.F90:83-94 (1-based in the
   reference, 0-based here) */
enum {
  Vy_xmin = 0, Vz_xmin, Vy_xmax, Vz_xmax, Vx_ymin, Vz_ymin,
  Vx_ymax, Vz_ymax, Vx_zmin, Vy_zmin, Vx_zmax, Vy_zmax
};
/* PML paper notation, SRC/TLM_MODULES/PML_module.F90:59-70 */
enum {
  Vxny = 0, Vxnz, Vxpy, Vxpz, Vynx, Vynz, Vypx, Vypz, Vznx, Vzny, Vzpx, Vzpy
};
/* field components, SRC/TLM_MODULES/TLM_Modules.F90:164-176 (0-based) */
enum { Ex = 0, Ey, Ez, Hx, Hy, Hz, Jx, Jy, Jz, Mx, My, Mz };

typedef struct {
  double Vxt, Vyt, Vzt, Ix, Iy, Iz, Ixt, Iyt, Izt;
  double Vi[12];
  double Vyxt, Vzxt, Vxyt, Vzyt, Vyzt, Vxzt;
} pml_cell_t; /* PML_data_type, PML_module.F90:116-128 */

/* PML_material_data_type (PML_module.F90:131-155): the values one step older
   than those in pml_cell_t, plus the capacitive / inductive stub state.
   Index 0,1,2 = x,y,z.  The reference also stores Ix_m1.. and Vyxt_m1..,
   which its update never reads; they are left out. */
typedef struct {
  double Vt_m1[3];   /* Vxt_m1, Vyt_m1, Vzt_m1 */
  double It_m1[3];   /* Ixt_m1, Iyt_m1, Izt_m1 */
  double Vi_m1[12];
  double Vosr[3], Vos[3], Vos_m1[3];
  double Vssr[3];
  double Vs[3], Vs_m1[3];
  double Vc[3], Vc_m1[3];
} pml_mat_t;

typedef struct {
  int order;
  double f;
  double w[ORACLE_MAX_ORDER + 1];
} zresp_t; /* Zfilter_response, FILTER/filter_types.F90:56-62 */

struct tlm_oracle_state {
  tlm_oracle_problem p;
  int nx, ny, nz;
  double *V;
  int32_t timestep; /* last completed timestep */
  int32_t *sp_filter;  /* cell_update_code_to_material_data(:,2), 1-based */
  zresp_t *eps_f, *mu_f;
  pml_cell_t *pml;
  pml_mat_t *pml_mat;  /* PML cells inside a volume material, traversal order */
  int32_t *pml_mat_pos; /* PML_material_array_pos per PML cell, 1-based or 0 */
  double *face_probe_rec; /* [n_timesteps][n_face_probes] */
  double *ff_acc;         /* far field, per surface face: J(3), M(3) complex */
  double *cell_exc;    /* [n_exc_cells][9] */
  int32_t *cell_exc_type; /* [n_exc_cells][6] */
  double *cell_out;    /* [n_out_cells][6] */
  double *face_exc;    /* [n_exc_faces][2][12] */
  int32_t *face_exc_type; /* [n_exc_faces][2][6] */
  double *face_out;    /* [n_out_faces][2][6] */
  int32_t *face_code;  /* [nz][ny][nx][3] -> 1-based special face index */
  double *dft;         /* per surface face: re, im */
  int32_t *dft_off;
  /* host threads for scatter and connect (tlm_oracle_set_threads), and the
     running output / excitation counters at the start of every z-plane, so
     the planes can be taken by different threads with the numbering of the
     sequential traversal */
  int threads;
  int32_t *plane_out0, *plane_exc0, *plane_fexc0, *plane_fout0;
  /* thin-layer filter responses: per special face two polarisations of
     four filters (Z11, Z12, Z21, Z22), allocate_surface_material_filter_data */
  zresp_t *sm_f;
  int err;
};

#define VIDX(s, port, cx, cy, cz) \
  ((((size_t)(cz) * ((s)->ny + 2) + (size_t)(cy)) * ((s)->nx + 2) + (size_t)(cx)) * 12 + (port))
#define V_(port, cx, cy, cz) s->V[VIDX(s, port, cx, cy, cz)]

static int nint(double x) { return (int)lround(x); } /* Fortran NINT */

/* evaluate_Zfilter, FILTER/filter_subroutines.F90:510-540 */
static void evaluate_Zfilter(const double *a, const double *b, zresp_t *ft, double G) {
  double W0 = G;
  for (int i = 1; i <= ft->order; i++) W0 = W0 - b[i] * ft->w[i];
  W0 = W0 / b[0];
  ft->w[0] = W0;
  double F0 = 0.0;
  for (int i = 0; i <= ft->order; i++) F0 = F0 + a[i] * ft->w[i];
  ft->f = F0;
}

/* timeshift_Zfilter, FILTER/filter_subroutines.F90:557-575 */
static void timeshift_Zfilter(zresp_t *ft) {
  for (int i = ft->order; i >= 1; i--) ft->w[i] = ft->w[i - 1];
}

/* add_shunt_admittance / add_series_impedance, scatter.F90:606-661 */
static void add_shunt_admittance(double *V1, double *Y1, double V2, double Y2) {
  double V = (*V1 * *Y1 + V2 * Y2) / (*Y1 + Y2);
  double Y = *Y1 + Y2;
  *V1 = V;
  *Y1 = Y;
}
static void add_series_impedance(double *V1, double *Z1, double V2, double Z2) {
  double V = *V1 + V2;
  double Z = *Z1 + Z2;
  *V1 = V;
  *Z1 = Z;
}

tlm_oracle_state *tlm_oracle_create(const tlm_oracle_problem *p) {
  tlm_oracle_state *s = (tlm_oracle_state *)calloc(1, sizeof(*s));
  if (!s) return NULL;
  s->p = *p;
  s->nx = p->nx;
  s->ny = p->ny;
  s->nz = p->nz;
  size_t nV = (size_t)(p->nx + 2) * (p->ny + 2) * (p->nz + 2) * 12;
  s->V = (double *)calloc(nV, sizeof(double)); /* allocate_mesh.F90:120, V=0 */

  /* allocate_volume_material_filter_data, TLM_volume_materials.F90:401-518 */
  s->sp_filter = (int32_t *)calloc((size_t)p->n_special + 1, sizeof(int32_t));
  int storage = 0;
  for (int c = 0; c < p->n_special; c++) {
    int m = p->sp_material[c];
    if (m != 0 && p->mat_type[m - 1] == 3) {
      s->sp_filter[c] = storage + 1;
      storage += 3;
    }
  }
  s->eps_f = (zresp_t *)calloc((size_t)storage + 1, sizeof(zresp_t));
  s->mu_f = (zresp_t *)calloc((size_t)storage + 1, sizeof(zresp_t));
  for (int c = 0; c < p->n_special; c++) {
    int m = p->sp_material[c];
    if (s->sp_filter[c]) {
      for (int k = 0; k < 3; k++) {
        s->eps_f[s->sp_filter[c] - 1 + k].order = p->mat_eps_order[m - 1];
        s->mu_f[s->sp_filter[c] - 1 + k].order = p->mat_mu_order[m - 1];
      }
    }
  }
  s->pml = (pml_cell_t *)calloc((size_t)p->n_pml_cells + 1, sizeof(pml_cell_t));
  s->face_probe_rec = (double *)calloc((size_t)p->n_timesteps * p->n_face_probes + 1, sizeof(double));
  s->ff_acc = (double *)calloc((size_t)(p->n_ff ? p->ff_face_ptr[p->n_ff] : 0) * 12 + 1, sizeof(double));
  /* allocate_PML_material_data, TLM_PML_volume_materials.F90:590-740: a
     PML cell whose special cell has a DISPERSIVE-type material gets the next
     PML material record, in special-cell (traversal) order; all zero */
  s->pml_mat_pos = (int32_t *)calloc((size_t)p->n_pml_cells + 1, sizeof(int32_t));
  {
    int n_pm = 0;
    for (int c = 0; c < p->n_special; c++) {
      int pc = p->sp_pml[c], m = p->sp_material[c];
      if (pc && m && p->mat_type[m - 1] == 3) s->pml_mat_pos[pc - 1] = ++n_pm;
    }
    s->pml_mat = (pml_mat_t *)calloc((size_t)n_pm + 1, sizeof(pml_mat_t));
  }
  s->cell_exc = (double *)calloc((size_t)p->n_exc_cells * 9 + 1, sizeof(double));
  s->cell_exc_type = (int32_t *)calloc((size_t)p->n_exc_cells * 6 + 1, sizeof(int32_t));
  for (int i = 0; i < p->n_exc_cells * 6; i++) s->cell_exc_type[i] = 1; /* soft, set_update_codes.F90:195 */
  s->cell_out = (double *)calloc((size_t)p->n_out_cells * 6 + 1, sizeof(double));
  s->face_exc = (double *)calloc((size_t)p->n_exc_faces * 24 + 1, sizeof(double));
  s->face_exc_type = (int32_t *)calloc((size_t)p->n_exc_faces * 12 + 1, sizeof(int32_t));
  for (int i = 0; i < p->n_exc_faces * 12; i++) s->face_exc_type[i] = 1; /* set_update_codes.F90:593 */
  s->face_out = (double *)calloc((size_t)p->n_out_faces * 12 + 1, sizeof(double));
  s->face_code = (int32_t *)calloc((size_t)p->nx * p->ny * p->nz * 3, sizeof(int32_t));
  for (int f = 0; f < p->n_faces; f++) {
    size_t cell = ((size_t)(p->face_cz[f] - 1) * p->ny + (p->face_cy[f] - 1)) * p->nx + (p->face_cx[f] - 1);
    s->face_code[cell * 3 + (p->face_dir[f] - 1)] = f + 1;
  }
  s->sm_f = (zresp_t *)calloc((size_t)p->n_faces * 8 + 1, sizeof(zresp_t));
  for (int f = 0; f < p->n_faces; f++) {
    int sm = p->face_smat ? p->face_smat[f] : 0;
    if (!sm || !p->face_mat || p->face_mat[f] != 3) continue;
    int m = abs(sm) - 1, d = p->face_dir[f];
    int pols[2] = {d == 1 ? 1 : 0, d == 3 ? 1 : 2}; /* x faces: y, z; y faces: x, z; z faces: x, y */
    for (int q = 0; q < 2; q++)
      for (int k = 0; k < 4; k++) s->sm_f[((size_t)f * 2 + q) * 4 + k].order = p->smat_order[(m * 3 + pols[q]) * 4 + k];
  }
  s->threads = 1;
  s->plane_out0 = (int32_t *)calloc((size_t)p->nz + 1, sizeof(int32_t));
  s->plane_exc0 = (int32_t *)calloc((size_t)p->nz + 1, sizeof(int32_t));
  s->plane_fexc0 = (int32_t *)calloc((size_t)p->nz + 1, sizeof(int32_t));
  s->plane_fout0 = (int32_t *)calloc((size_t)p->nz + 1, sizeof(int32_t));
  {
    /* the counters scatter() and connect() advance, at the start of each plane */
    int out = 0, exc = 0, fexc = 0, fout = 0;
    size_t cell = 0;
    for (int cz = 0; cz < p->nz; cz++) {
      s->plane_out0[cz] = out; s->plane_exc0[cz] = exc;
      s->plane_fexc0[cz] = fexc; s->plane_fout0[cz] = fout;
      for (size_t c = 0; c < (size_t)p->nx * p->ny; c++, cell++) {
        int code = p->cell_code[cell];
        if (code) {
          int sc = code - 1;
          if (p->sp_output[sc]) out++;
          if (!p->sp_pml[sc] && p->sp_excitation[sc]) exc++;
        }
        /* connect() skips the faces on the mesh's min boundary planes */
        const int on_min[3] = {(int)(c % (size_t)p->nx) == 0, (int)(c / (size_t)p->nx) == 0, cz == 0};
        for (int d = 0; d < 3; d++) {
          int f = on_min[d] ? 0 : s->face_code[cell * 3 + d];
          if (f) {
            if (p->face_exc[f - 1]) fexc++;
            if (p->face_out[f - 1]) fout++;
          }
        }
      }
    }
  }
  int ndftf = p->n_dft ? p->dft_face_ptr[p->n_dft] : 0;
  s->dft = (double *)calloc((size_t)ndftf * 2 + 1, sizeof(double));
  s->timestep = 0;
  return s;
}

void tlm_oracle_destroy(tlm_oracle_state *s) {
  if (!s) return;
  free(s->V); free(s->sp_filter); free(s->eps_f); free(s->mu_f); free(s->pml); free(s->pml_mat); free(s->pml_mat_pos); free(s->face_probe_rec); free(s->ff_acc);
  free(s->cell_exc); free(s->cell_exc_type); free(s->cell_out); free(s->face_exc);
  free(s->face_exc_type); free(s->face_out); free(s->face_code); free(s->dft);
  free(s->plane_out0); free(s->plane_exc0); free(s->plane_fexc0); free(s->plane_fout0);
  free(s->sm_f);
  free(s);
}

/* get_interpolated_excitation_value, EXCITATION/excitation.F90:645-690 */
static double interp_face_value(const tlm_oracle_state *s, double offset, int timestep) {
  const tlm_oracle_problem *p = &s->p;
  double t_offset = (offset - p->hs_offset_min) / p->hs_c;
  double local_time = ((double)(timestep - 1)) * p->dt - t_offset;
  int ts1 = nint(local_time / p->dt);
  int ts2 = ts1 + 1;
  double delta_t = local_time - (double)ts1 * p->dt;
  const double *vf = p->fn_value_face + (size_t)(p->hs_fn - 1) * p->n_timesteps;
  double v1 = (ts1 >= 1 && ts1 <= p->n_timesteps) ? vf[ts1 - 1] : 0.0;
  double v2 = (ts2 >= 1 && ts2 <= p->n_timesteps) ? vf[ts2 - 1] : 0.0;
  return v1 + delta_t * (v2 - v1) / p->dt;
}

/* excitation(), EXCITATION/excitation.F90:578-626 with Point_excitation
   (excitation_points.F90:231-335, centre points) and
   Huygens_surface_excitation (huygens_surface.F90:734-848) */
static void excitation(tlm_oracle_state *s, int timestep) {
  const tlm_oracle_problem *p = &s->p;
  memset(s->cell_exc, 0, sizeof(double) * (size_t)p->n_exc_cells * 9);
  memset(s->face_exc, 0, sizeof(double) * (size_t)p->n_exc_faces * 24);
  for (int e = 0; e < p->n_exc_points; e++) {
    int cell = p->pt_cell[e] - 1, comp = p->pt_comp[e] - 1;
    double value = p->fn_value[(size_t)(p->pt_fn[e] - 1) * p->n_timesteps + (timestep - 1)];
    s->cell_exc[cell * 9 + comp] = s->cell_exc[cell * 9 + comp] + value;
    if (comp < 6) s->cell_exc_type[cell * 6 + comp] = p->pt_type[e];
  }
  /* Point_excitation, face points (excitation_points.F90:286-323): the value
     goes to both sides of the face, the source type too (components 1..6);
     then Surface_excitation (excitation_surfaces.F90:218-275), whose faces
     follow the points in the list: one side, or both; Mode_excitation's
     faces (mode_excitation.F90:370-415) come last, each value times its
     mode field (E and H only, so the Huygens J, M added below are not
     reordered against them) */
  for (int e = 0; e < p->n_face_points; e++) {
    int face = p->fpt_face[e] - 1, comp = p->fpt_comp[e] - 1;
    double value = p->fn_value_face[(size_t)(p->fpt_fn[e] - 1) * p->n_timesteps + (timestep - 1)];
    if (p->fpt_scale) value = p->fpt_scale[e] * value;
    int only = p->fpt_side ? p->fpt_side[e] : 0;
    for (int side = 0; side < 2; side++) {
      if (only && side != only - 1) continue;
      double *fe = s->face_exc + (size_t)face * 24 + side * 12;
      fe[comp] = fe[comp] + value;
      if (comp < 6) s->face_exc_type[(size_t)face * 12 + side * 6 + comp] = p->fpt_type[e];
    }
  }
  for (int h = 0; h < (p->hs_outer ? 0 : p->hs_n); h++) {
    double value = interp_face_value(s, p->hs_offset[h], timestep);
    double nxx = p->hs_norm[3 * h], nyy = p->hs_norm[3 * h + 1], nzz = p->hs_norm[3 * h + 2];
    const double *Hi = p->hs_Hi, *Ei = p->hs_Ei;
    double Js[3], Ms[3];
    Js[0] = (nyy * value * (Hi[2]) - nzz * value * (Hi[1]));
    Js[1] = (nzz * value * (Hi[0]) - nxx * value * (Hi[2]));
    Js[2] = (nxx * value * (Hi[1]) - nyy * value * (Hi[0]));
    Ms[0] = -(nyy * value * (Ei[2]) - nzz * value * (Ei[1]));
    Ms[1] = -(nzz * value * (Ei[0]) - nxx * value * (Ei[2]));
    Ms[2] = -(nxx * value * (Ei[1]) - nyy * value * (Ei[0]));
    double *fe = s->face_exc + (size_t)(p->hs_face_exc[h] - 1) * 24;
    for (int side = 0; side < 2; side++) {
      for (int k = 0; k < 3; k++) {
        fe[side * 12 + Jx + k] = fe[side * 12 + Jx + k] + Js[k];
        fe[side * 12 + Mx + k] = fe[side * 12 + Mx + k] + Ms[k];
      }
    }
  }
}

/* scatter_PML.F90:22-313 (free-space PML cell) */
static void scatter_pml_cell(tlm_oracle_state *s, int cx, int cy, int cz, int pml_cell, int output, int *output_cell_number) {
  const tlm_oracle_problem *p = &s->p;
  const double *P = p->pml_params + (size_t)(p->pml_cell_param[pml_cell - 1] - 1) * 15;
  double ax = P[0], ay = P[1], az = P[2];
  double exp_x = P[3], exp_y = P[4], exp_z = P[5];
  double Csx = P[6], Csy = P[7], Csz = P[8];
  double Csx2 = P[9], Csy2 = P[10], Csz2 = P[11];
  double Csy_sz = P[12], Csz_sx = P[13], Csx_sy = P[14];
  double exp_xi = exp_x, exp_yi = exp_y, exp_zi = exp_z;
  double exp_xr = exp_x, exp_yr = exp_y, exp_zr = exp_z;
  pml_cell_t *pc = &s->pml[pml_cell - 1];

  double last_Ix = pc->Ix, last_Iy = pc->Iy, last_Iz = pc->Iz;
  double last_Vi[12];
  memcpy(last_Vi, pc->Vi, sizeof(last_Vi));
  double last_Vxt = pc->Vxt, last_Vyt = pc->Vyt, last_Vzt = pc->Vzt;
  double last_Vyxt = pc->Vyxt, last_Vzxt = pc->Vzxt, last_Vxyt = pc->Vxyt;
  double last_Vzyt = pc->Vzyt, last_Vyzt = pc->Vyzt, last_Vxzt = pc->Vxzt;

  /* STAGE 3 */
  V_(Vynx, cx, cy, cz) = V_(Vynx, cx, cy, cz) * exp_yi;
  V_(Vypx, cx, cy, cz) = V_(Vypx, cx, cy, cz) * exp_yi;
  V_(Vznx, cx, cy, cz) = V_(Vznx, cx, cy, cz) * exp_zi;
  V_(Vzpx, cx, cy, cz) = V_(Vzpx, cx, cy, cz) * exp_zi;
  V_(Vxny, cx, cy, cz) = V_(Vxny, cx, cy, cz) * exp_xi;
  V_(Vxpy, cx, cy, cz) = V_(Vxpy, cx, cy, cz) * exp_xi;
  V_(Vzny, cx, cy, cz) = V_(Vzny, cx, cy, cz) * exp_zi;
  V_(Vzpy, cx, cy, cz) = V_(Vzpy, cx, cy, cz) * exp_zi;
  V_(Vxnz, cx, cy, cz) = V_(Vxnz, cx, cy, cz) * exp_xi;
  V_(Vxpz, cx, cy, cz) = V_(Vxpz, cx, cy, cz) * exp_xi;
  V_(Vynz, cx, cy, cz) = V_(Vynz, cx, cy, cz) * exp_yi;
  V_(Vypz, cx, cy, cz) = V_(Vypz, cx, cy, cz) * exp_yi;

  /* STAGE 4 */
  double Vx = (V_(Vynx, cx, cy, cz) + V_(Vypx, cx, cy, cz) + V_(Vznx, cx, cy, cz) + V_(Vzpx, cx, cy, cz)) / 2.0;
  double Vy = (V_(Vxny, cx, cy, cz) + V_(Vxpy, cx, cy, cz) + V_(Vzny, cx, cy, cz) + V_(Vzpy, cx, cy, cz)) / 2.0;
  double Vz = (V_(Vxnz, cx, cy, cz) + V_(Vxpz, cx, cy, cz) + V_(Vynz, cx, cy, cz) + V_(Vypz, cx, cy, cz)) / 2.0;
  double Ix = (V_(Vypz, cx, cy, cz) - V_(Vzpy, cx, cy, cz) - V_(Vynz, cx, cy, cz) + V_(Vzny, cx, cy, cz)) / (2.0 * Z0);
  double Iy = (V_(Vzpx, cx, cy, cz) - V_(Vxpz, cx, cy, cz) - V_(Vznx, cx, cy, cz) + V_(Vxnz, cx, cy, cz)) / (2.0 * Z0);
  double Iz = (V_(Vxpy, cx, cy, cz) - V_(Vypx, cx, cy, cz) - V_(Vxny, cx, cy, cz) + V_(Vynx, cx, cy, cz)) / (2.0 * Z0);

  /* STAGE 5 */
  double Vx_PML_shunt = ax * (-(last_Vi[Vznx] + last_Vi[Vzpx] + last_Vi[Vynx] + last_Vi[Vypx]) / 2.0
                              + Csy * ((V_(Vznx, cx, cy, cz) + V_(Vzpx, cx, cy, cz)) + (last_Vi[Vznx] + last_Vi[Vzpx]))
                              + Csz * ((V_(Vynx, cx, cy, cz) + V_(Vypx, cx, cy, cz)) + (last_Vi[Vynx] + last_Vi[Vypx]))
                              + Csy_sz * last_Vxt);
  double Vy_PML_shunt = ay * (-(last_Vi[Vxny] + last_Vi[Vxpy] + last_Vi[Vzny] + last_Vi[Vzpy]) / 2.0
                              + Csz * ((V_(Vxny, cx, cy, cz) + V_(Vxpy, cx, cy, cz)) + (last_Vi[Vxny] + last_Vi[Vxpy]))
                              + Csx * ((V_(Vzny, cx, cy, cz) + V_(Vzpy, cx, cy, cz)) + (last_Vi[Vzny] + last_Vi[Vzpy]))
                              + Csz_sx * last_Vyt);
  double Vz_PML_shunt = az * (-(last_Vi[Vynz] + last_Vi[Vypz] + last_Vi[Vxnz] + last_Vi[Vxpz]) / 2.0
                              + Csx * ((V_(Vynz, cx, cy, cz) + V_(Vypz, cx, cy, cz)) + (last_Vi[Vynz] + last_Vi[Vypz]))
                              + Csy * ((V_(Vxnz, cx, cy, cz) + V_(Vxpz, cx, cy, cz)) + (last_Vi[Vxnz] + last_Vi[Vxpz]))
                              + Csx_sy * last_Vzt);
  /* STAGE 6 */
  double Vxt = ax * Vx + Vx_PML_shunt;
  double Vyt = ay * Vy + Vy_PML_shunt;
  double Vzt = az * Vz + Vz_PML_shunt;
  /* STAGE 7a */
  double Ixt = 0, Iyt = 0, Izt = 0;
  if (output) {
    double last_Ixt = pc->Ixt, last_Iyt = pc->Iyt, last_Izt = pc->Izt;
    Ixt = ax * (Ix - last_Ix + Csx2 * (Ix + last_Ix) + Csy_sz * last_Ixt);
    Iyt = ay * (Iy - last_Iy + Csy2 * (Iy + last_Iy) + Csz_sx * last_Iyt);
    Izt = az * (Iz - last_Iz + Csz2 * (Iz + last_Iz) + Csx_sy * last_Izt);
  }
  /* STAGE 7 */
  double Vxy_PML_series = az * (Z0 * (-last_Iz + Csy2 * (Iz + last_Iz)) + Csx_sy * last_Vxyt);
  double Vyx_PML_series = az * (Z0 * (-last_Iz + Csx2 * (Iz + last_Iz)) + Csx_sy * last_Vyxt);
  double Vzx_PML_series = ay * (Z0 * (-last_Iy + Csx2 * (Iy + last_Iy)) + Csz_sx * last_Vzxt);
  double Vxz_PML_series = ay * (Z0 * (-last_Iy + Csz2 * (Iy + last_Iy)) + Csz_sx * last_Vxzt);
  double Vyz_PML_series = ax * (Z0 * (-last_Ix + Csz2 * (Ix + last_Ix)) + Csy_sz * last_Vyzt);
  double Vzy_PML_series = ax * (Z0 * (-last_Ix + Csy2 * (Ix + last_Ix)) + Csy_sz * last_Vzyt);
  /* STAGE 8 */
  double Vxyt = az * Iz * Z0 + Vxy_PML_series;
  double Vyxt = az * Iz * Z0 + Vyx_PML_series;
  double Vzxt = ay * Iy * Z0 + Vzx_PML_series;
  double Vxzt = ay * Iy * Z0 + Vxz_PML_series;
  double Vyzt = ax * Ix * Z0 + Vyz_PML_series;
  double Vzyt = ax * Ix * Z0 + Vzy_PML_series;
  /* STAGE 9 */
  pc->Ix = Ix; pc->Iy = Iy; pc->Iz = Iz;
  for (int k = 0; k < 12; k++) pc->Vi[k] = V_(k, cx, cy, cz);
  pc->Vxt = Vxt; pc->Vyt = Vyt; pc->Vzt = Vzt;
  if (output) { pc->Ixt = Ixt; pc->Iyt = Iyt; pc->Izt = Izt; }
  pc->Vxyt = Vxyt; pc->Vyxt = Vyxt; pc->Vzxt = Vzxt; pc->Vxzt = Vxzt; pc->Vzyt = Vzyt; pc->Vyzt = Vyzt;
  /* STAGE 10 */
  double Vynx_PML = Vx_PML_shunt - Vyx_PML_series;
  double Vypx_PML = Vx_PML_shunt + Vyx_PML_series;
  double Vznx_PML = Vx_PML_shunt + Vzx_PML_series;
  double Vzpx_PML = Vx_PML_shunt - Vzx_PML_series;
  double Vxny_PML = Vy_PML_shunt + Vxy_PML_series;
  double Vxpy_PML = Vy_PML_shunt - Vxy_PML_series;
  double Vzny_PML = Vy_PML_shunt - Vzy_PML_series;
  double Vzpy_PML = Vy_PML_shunt + Vzy_PML_series;
  double Vynz_PML = Vz_PML_shunt + Vyz_PML_series;
  double Vypz_PML = Vz_PML_shunt - Vyz_PML_series;
  double Vxnz_PML = Vz_PML_shunt - Vxz_PML_series;
  double Vxpz_PML = Vz_PML_shunt + Vxz_PML_series;
  /* STAGE 11 */
  double V_max, V_min;
  V_max = V_(Vypx, cx, cy, cz); V_min = V_(Vynx, cx, cy, cz);
  V_(Vynx, cx, cy, cz) = ax * Vx - az * Z0 * Iz - V_max + Vynx_PML;
  V_(Vypx, cx, cy, cz) = ax * Vx + az * Z0 * Iz - V_min + Vypx_PML;
  V_max = V_(Vzpx, cx, cy, cz); V_min = V_(Vznx, cx, cy, cz);
  V_(Vznx, cx, cy, cz) = ax * Vx + ay * Z0 * Iy - V_max + Vznx_PML;
  V_(Vzpx, cx, cy, cz) = ax * Vx - ay * Z0 * Iy - V_min + Vzpx_PML;
  V_max = V_(Vzpy, cx, cy, cz); V_min = V_(Vzny, cx, cy, cz);
  V_(Vzny, cx, cy, cz) = ay * Vy - ax * Z0 * Ix - V_max + Vzny_PML;
  V_(Vzpy, cx, cy, cz) = ay * Vy + ax * Z0 * Ix - V_min + Vzpy_PML;
  V_max = V_(Vxpy, cx, cy, cz); V_min = V_(Vxny, cx, cy, cz);
  V_(Vxny, cx, cy, cz) = ay * Vy + az * Z0 * Iz - V_max + Vxny_PML;
  V_(Vxpy, cx, cy, cz) = ay * Vy - az * Z0 * Iz - V_min + Vxpy_PML;
  V_max = V_(Vxpz, cx, cy, cz); V_min = V_(Vxnz, cx, cy, cz);
  V_(Vxnz, cx, cy, cz) = az * Vz - ay * Z0 * Iy - V_max + Vxnz_PML;
  V_(Vxpz, cx, cy, cz) = az * Vz + ay * Z0 * Iy - V_min + Vxpz_PML;
  V_max = V_(Vypz, cx, cy, cz); V_min = V_(Vynz, cx, cy, cz);
  V_(Vynz, cx, cy, cz) = az * Vz + ax * Z0 * Ix - V_max + Vynz_PML;
  V_(Vypz, cx, cy, cz) = az * Vz - ax * Z0 * Ix - V_min + Vypz_PML;
  /* STAGE 12 */
  if (output) {
    double dl = p->dl;
    double *f = s->cell_out + (size_t)(*output_cell_number) * 6;
    (*output_cell_number)++;
    f[Ex] = -Vxt / dl; f[Ey] = -Vyt / dl; f[Ez] = -Vzt / dl;
    f[Hx] = Ixt / dl; f[Hy] = Iyt / dl; f[Hz] = Izt / dl;
  }
  /* STAGE 13 */
  V_(Vynx, cx, cy, cz) = V_(Vynx, cx, cy, cz) * exp_yr;
  V_(Vypx, cx, cy, cz) = V_(Vypx, cx, cy, cz) * exp_yr;
  V_(Vznx, cx, cy, cz) = V_(Vznx, cx, cy, cz) * exp_zr;
  V_(Vzpx, cx, cy, cz) = V_(Vzpx, cx, cy, cz) * exp_zr;
  V_(Vxny, cx, cy, cz) = V_(Vxny, cx, cy, cz) * exp_xr;
  V_(Vxpy, cx, cy, cz) = V_(Vxpy, cx, cy, cz) * exp_xr;
  V_(Vzny, cx, cy, cz) = V_(Vzny, cx, cy, cz) * exp_zr;
  V_(Vzpy, cx, cy, cz) = V_(Vzpy, cx, cy, cz) * exp_zr;
  V_(Vxnz, cx, cy, cz) = V_(Vxnz, cx, cy, cz) * exp_xr;
  V_(Vxpz, cx, cy, cz) = V_(Vxpz, cx, cy, cz) * exp_xr;
  V_(Vynz, cx, cy, cz) = V_(Vynz, cx, cy, cz) * exp_yr;
  V_(Vypz, cx, cy, cz) = V_(Vypz, cx, cy, cz) * exp_yr;
}

/* PML cell inside a non-dispersive volume material,
   TLM_SOLVER/scatter_PML_material.F90:22-534.  Second-order recursions in
   time for the stretched voltages (with the capacitive stub), the stretched
   currents (with the inductive stub) and the series PML terms; the
   coefficients are rebuilt from sx,sy,sz and the material every call, as the
   reference does.  Axis a = x,y,z has partners (j,k) = (y,z),(z,x),(x,y). */
static void scatter_pml_material_cell(tlm_oracle_state *s, int cx, int cy, int cz, int pml_cell, int material_number,
                                      int output, int *output_cell_number) {
  const tlm_oracle_problem *p = &s->p;
  const int prow = p->pml_cell_param[pml_cell - 1] - 1;
  const double *P = p->pml_params + (size_t)prow * 15;
  const double *S = p->pml_sigma + (size_t)prow * 3;
  const int m = material_number - 1;
  const double dt = p->dt;
  pml_cell_t *pc = &s->pml[pml_cell - 1];
  pml_mat_t *pm = &s->pml_mat[s->pml_mat_pos[pml_cell - 1] - 1];

  /* STAGE 1 (:24-221): the same Ys, Ge, Zs, Rm on the three axes */
  const double Ys = p->mat_Ys_eps_f[m] / Y0, Ge = p->mat_Ge[m] / Y0;
  const double Zs = p->mat_Zs_mu_f[m], Rm = p->mat_Rm[m];
  const double sg[3] = {S[0], S[1], S[2]};
  const double ex[3] = {P[3], P[4], P[5]}; /* exp_x, exp_y, exp_z */
  double A[3][3], B[3][3], Cc[3][3], D[3][3], Sc[3][3], T[3][3], Pc[3][3], Q[3][3];
  for (int a = 0; a < 3; a++) {
    const double sj = sg[(a + 1) % 3], sk = sg[(a + 2) % 3], sa = sg[a];
    const double GpY2 = (Ge + Ys) / 2.0;
    A[a][0] = 8.0 + 4.0 * GpY2 + 2.0 * dt * (sj + sk) * (1.0 + GpY2) + dt * dt * sj * sk * GpY2;
    A[a][1] = -2.0 * (8.0 + 4.0 * GpY2) + 2.0 * (dt * dt * sj * sk * GpY2);
    A[a][2] = 8.0 + 4.0 * GpY2 - 2.0 * dt * (sj + sk) * (1.0 + GpY2) + dt * dt * sj * sk * GpY2;
    B[a][0] = 4.0 + 2.0 * dt * sj; B[a][1] = -8.0; B[a][2] = 4.0 - 2.0 * dt * sj;
    Cc[a][0] = 4.0 + 2.0 * dt * sk; Cc[a][1] = -8.0; Cc[a][2] = 4.0 - 2.0 * dt * sk;
    D[a][0] = 4.0 * Ys + 2.0 * dt * (sj + sk) * Ys + 1.0 * (dt * dt * sj * sk * Ys);
    D[a][1] = -8.0 * Ys + 2.0 * (dt * dt * sj * sk * Ys);
    D[a][2] = 4.0 * Ys - 2.0 * dt * (sj + sk) * Ys + 1.0 * (dt * dt * sj * sk * Ys);
    const double ZpR = Zs + Rm;
    Sc[a][0] = 16.0 * Z0 + 4.0 * ZpR + 2.0 * dt * (sj + sk) * (2.0 * Z0 + ZpR) + dt * dt * sj * sk * ZpR;
    Sc[a][1] = -32.0 * Z0 - 8.0 * ZpR + 2.0 * dt * dt * sj * sk * ZpR;
    Sc[a][2] = 16.0 * Z0 + 4.0 * ZpR - 2.0 * dt * (sj + sk) * (2.0 * Z0 + ZpR) + dt * dt * sj * sk * ZpR;
    T[a][0] = 8.0 + 4.0 * dt * sa; T[a][1] = -16.0; T[a][2] = 8.0 - 4.0 * dt * sa;
    Pc[a][0] = 4.0 + 2.0 * dt * sa; Pc[a][1] = -8.0; Pc[a][2] = 4.0 - 2.0 * dt * sa;
    Q[a][0] = 4.0 * Zs + 2.0 * dt * (sj + sk) * Zs + 1.0 * (dt * dt * sj * sk * Zs);
    Q[a][1] = -8.0 * Zs + 2.0 * (dt * dt * sj * sk * Zs);
    Q[a][2] = 4.0 * Zs - 2.0 * dt * (sj + sk) * Zs + 1.0 * (dt * dt * sj * sk * Zs);
  }
  /* series terms V_{ab}t: U uses the third axis c, W the axis b (:169-195) */
  const int sab[6][2] = {{0, 1}, {1, 0}, {1, 2}, {2, 1}, {2, 0}, {0, 2}}; /* xy yx yz zy zx xz */
  double U0[6], U1[6], W0[6], W1[6];
  for (int q = 0; q < 6; q++) {
    const int a = sab[q][0], b = sab[q][1], c = 3 - a - b;
    U0[q] = 2.0 + dt * sg[c];
    U1[q] = -2.0 + dt * sg[c];
    W0[q] = Z0 * (2.0 + dt * sg[b]);
    W1[q] = Z0 * (-2.0 + dt * sg[b]);
  }

  /* STAGE 2: previous values */
  double Vi_m1[12], Vi_m2[12];
  memcpy(Vi_m1, pc->Vi, sizeof(Vi_m1));
  memcpy(Vi_m2, pm->Vi_m1, sizeof(Vi_m2));
  const double Vt_m1[3] = {pc->Vxt, pc->Vyt, pc->Vzt};
  const double It_m1[3] = {pc->Ixt, pc->Iyt, pc->Izt};
  const double It_m2[3] = {pm->It_m1[0], pm->It_m1[1], pm->It_m1[2]};
  const double Vabt_m1[6] = {pc->Vxyt, pc->Vyxt, pc->Vyzt, pc->Vzyt, pc->Vzxt, pc->Vxzt};
  double Vos[3], Vss[3];
  for (int a = 0; a < 3; a++) {
    Vos[a] = pm->Vosr[a];  /* capacitive stub incident = last reflected */
    Vss[a] = -pm->Vssr[a]; /* inductive stub incident = -last reflected */
  }

  /* STAGE 3: half-cell loss on the incident pulses */
  V_(Vynx, cx, cy, cz) = V_(Vynx, cx, cy, cz) * ex[1];
  V_(Vypx, cx, cy, cz) = V_(Vypx, cx, cy, cz) * ex[1];
  V_(Vznx, cx, cy, cz) = V_(Vznx, cx, cy, cz) * ex[2];
  V_(Vzpx, cx, cy, cz) = V_(Vzpx, cx, cy, cz) * ex[2];
  V_(Vxny, cx, cy, cz) = V_(Vxny, cx, cy, cz) * ex[0];
  V_(Vxpy, cx, cy, cz) = V_(Vxpy, cx, cy, cz) * ex[0];
  V_(Vzny, cx, cy, cz) = V_(Vzny, cx, cy, cz) * ex[2];
  V_(Vzpy, cx, cy, cz) = V_(Vzpy, cx, cy, cz) * ex[2];
  V_(Vxnz, cx, cy, cz) = V_(Vxnz, cx, cy, cz) * ex[0];
  V_(Vxpz, cx, cy, cz) = V_(Vxpz, cx, cy, cz) * ex[0];
  V_(Vynz, cx, cy, cz) = V_(Vynz, cx, cy, cz) * ex[1];
  V_(Vypz, cx, cy, cz) = V_(Vypz, cx, cy, cz) * ex[1];

  /* STAGE 4: stretched Vt.  Port pairs: B multiplies (x: z-ports on x faces,
     y: x-ports on y faces, z: y-ports on z faces), C the other pair */
  const int pb[3][2] = {{Vznx, Vzpx}, {Vxny, Vxpy}, {Vynz, Vypz}};
  const int pcp[3][2] = {{Vynx, Vypx}, {Vzny, Vzpy}, {Vxnz, Vxpz}};
  double Vt[3];
  for (int a = 0; a < 3; a++) {
    const int b0 = pb[a][0], b1 = pb[a][1], c0 = pcp[a][0], c1 = pcp[a][1];
    Vt[a] = (1.0 / A[a][0]) * (B[a][0] * (V_(b0, cx, cy, cz) + V_(b1, cx, cy, cz)) +
                               Cc[a][0] * (V_(c0, cx, cy, cz) + V_(c1, cx, cy, cz)) + D[a][0] * (Vos[a]) +
                               B[a][1] * (Vi_m1[b0] + Vi_m1[b1]) + Cc[a][1] * (Vi_m1[c0] + Vi_m1[c1]) +
                               D[a][1] * (pm->Vos[a]) + B[a][2] * (Vi_m2[b0] + Vi_m2[b1]) +
                               Cc[a][2] * (Vi_m2[c0] + Vi_m2[c1]) + D[a][2] * (pm->Vos_m1[a]) -
                               A[a][1] * Vt_m1[a] - A[a][2] * pm->Vt_m1[a]);
  }

  /* STAGE 5: stretched It through the series impedance */
  double Vc[3];
  Vc[0] = V_(Vypz, cx, cy, cz) - V_(Vzpy, cx, cy, cz) - V_(Vynz, cx, cy, cz) + V_(Vzny, cx, cy, cz) - Vss[0];
  Vc[1] = V_(Vzpx, cx, cy, cz) - V_(Vxpz, cx, cy, cz) - V_(Vznx, cx, cy, cz) + V_(Vxnz, cx, cy, cz) - Vss[1];
  Vc[2] = V_(Vxpy, cx, cy, cz) - V_(Vypx, cx, cy, cz) - V_(Vxny, cx, cy, cz) + V_(Vynx, cx, cy, cz) - Vss[2];
  double It[3];
  for (int a = 0; a < 3; a++)
    It[a] = (1.0 / Sc[a][0]) * (T[a][0] * Vc[a] + T[a][1] * pm->Vc[a] + T[a][2] * pm->Vc_m1[a] -
                                Sc[a][1] * It_m1[a] - Sc[a][2] * It_m2[a]);
  /* V_{ab}t is driven by the current of the third axis c */
  double Vabt[6];
  for (int q = 0; q < 6; q++) {
    const int c = 3 - sab[q][0] - sab[q][1];
    Vabt[q] = (1.0 / U0[q]) * (W0[q] * It[c] + W1[q] * It_m1[c] - U1[q] * Vabt_m1[q]);
  }
  const double Vxyt = Vabt[0], Vyxt = Vabt[1], Vyzt = Vabt[2], Vzyt = Vabt[3], Vzxt = Vabt[4], Vxzt = Vabt[5];

  /* STAGE 9: save for the next step */
  memcpy(pm->Vi_m1, pc->Vi, sizeof(pm->Vi_m1));
  for (int k = 0; k < 12; k++) pc->Vi[k] = V_(k, cx, cy, cz);
  for (int a = 0; a < 3; a++) {
    pm->Vt_m1[a] = Vt_m1[a];
    pm->It_m1[a] = It_m1[a];
    pm->Vc_m1[a] = pm->Vc[a];
    pm->Vc[a] = Vc[a];
  }
  pc->Vxt = Vt[0]; pc->Vyt = Vt[1]; pc->Vzt = Vt[2];
  pc->Ixt = It[0]; pc->Iyt = It[1]; pc->Izt = It[2];
  pc->Vxyt = Vxyt; pc->Vyxt = Vyxt; pc->Vyzt = Vyzt; pc->Vzyt = Vzyt; pc->Vzxt = Vzxt; pc->Vxzt = Vxzt;

  /* STAGE 11: scattered pulses */
  double V_max, V_min;
  V_max = V_(Vypx, cx, cy, cz); V_min = V_(Vynx, cx, cy, cz);
  V_(Vynx, cx, cy, cz) = Vt[0] - Vyxt - V_max;
  V_(Vypx, cx, cy, cz) = Vt[0] + Vyxt - V_min;
  V_max = V_(Vzpx, cx, cy, cz); V_min = V_(Vznx, cx, cy, cz);
  V_(Vznx, cx, cy, cz) = Vt[0] + Vzxt - V_max;
  V_(Vzpx, cx, cy, cz) = Vt[0] - Vzxt - V_min;
  V_max = V_(Vzpy, cx, cy, cz); V_min = V_(Vzny, cx, cy, cz);
  V_(Vzny, cx, cy, cz) = Vt[1] - Vzyt - V_max;
  V_(Vzpy, cx, cy, cz) = Vt[1] + Vzyt - V_min;
  V_max = V_(Vxpy, cx, cy, cz); V_min = V_(Vxny, cx, cy, cz);
  V_(Vxny, cx, cy, cz) = Vt[1] + Vxyt - V_max;
  V_(Vxpy, cx, cy, cz) = Vt[1] - Vxyt - V_min;
  V_max = V_(Vxpz, cx, cy, cz); V_min = V_(Vxnz, cx, cy, cz);
  V_(Vxnz, cx, cy, cz) = Vt[2] - Vxzt - V_max;
  V_(Vxpz, cx, cy, cz) = Vt[2] + Vxzt - V_min;
  V_max = V_(Vypz, cx, cy, cz); V_min = V_(Vynz, cx, cy, cz);
  V_(Vynz, cx, cy, cz) = Vt[2] + Vyzt - V_max;
  V_(Vypz, cx, cy, cz) = Vt[2] - Vyzt - V_min;

  /* capacitive stub scatter and history */
  for (int a = 0; a < 3; a++) {
    pm->Vosr[a] = Vt[a] - Vos[a];
    pm->Vos_m1[a] = pm->Vos[a];
    pm->Vos[a] = Vos[a];
  }
  /* inductive stub: voltage across the stub impedance, then its reflection */
  for (int a = 0; a < 3; a++) {
    const double Vs = (1.0 / Pc[a][0]) * (Q[a][0] * It[a] + Q[a][1] * It_m1[a] + Q[a][2] * It_m2[a] -
                                          Pc[a][1] * pm->Vs[a] - Pc[a][2] * pm->Vs_m1[a]);
    pm->Vssr[a] = (Vs + Vss[a]);
    pm->Vs_m1[a] = pm->Vs[a];
    pm->Vs[a] = Vs;
  }

  /* STAGE 12: output */
  if (output) {
    double dl = p->dl;
    double *f = s->cell_out + (size_t)(*output_cell_number) * 6;
    (*output_cell_number)++;
    f[Ex] = -Vt[0] / dl; f[Ey] = -Vt[1] / dl; f[Ez] = -Vt[2] / dl;
    f[Hx] = It[0] / dl; f[Hy] = It[1] / dl; f[Hz] = It[2] / dl;
  }

  /* STAGE 13: half-cell loss on the scattered pulses */
  V_(Vynx, cx, cy, cz) = V_(Vynx, cx, cy, cz) * ex[1];
  V_(Vypx, cx, cy, cz) = V_(Vypx, cx, cy, cz) * ex[1];
  V_(Vznx, cx, cy, cz) = V_(Vznx, cx, cy, cz) * ex[2];
  V_(Vzpx, cx, cy, cz) = V_(Vzpx, cx, cy, cz) * ex[2];
  V_(Vxny, cx, cy, cz) = V_(Vxny, cx, cy, cz) * ex[0];
  V_(Vxpy, cx, cy, cz) = V_(Vxpy, cx, cy, cz) * ex[0];
  V_(Vzny, cx, cy, cz) = V_(Vzny, cx, cy, cz) * ex[2];
  V_(Vzpy, cx, cy, cz) = V_(Vzpy, cx, cy, cz) * ex[2];
  V_(Vxnz, cx, cy, cz) = V_(Vxnz, cx, cy, cz) * ex[0];
  V_(Vxpz, cx, cy, cz) = V_(Vxpz, cx, cy, cz) * ex[0];
  V_(Vynz, cx, cy, cz) = V_(Vynz, cx, cy, cz) * ex[1];
  V_(Vypz, cx, cy, cz) = V_(Vypz, cx, cy, cz) * ex[1];
}

/* final scatter of the pulses, scatter.F90:519-547 (also :247-272) */
static void scatter_pulses(tlm_oracle_state *s, int cx, int cy, int cz, double Vx, double Vy, double Vz,
                           double Ix, double Iy, double Iz) {
  double V_min, V_max;
  V_min = V_(Vx_ymin, cx, cy, cz); V_max = V_(Vx_ymax, cx, cy, cz);
  V_(Vx_ymin, cx, cy, cz) = Vx - Z0 * Iz - V_max;
  V_(Vx_ymax, cx, cy, cz) = Vx + Z0 * Iz - V_min;
  V_min = V_(Vx_zmin, cx, cy, cz); V_max = V_(Vx_zmax, cx, cy, cz);
  V_(Vx_zmin, cx, cy, cz) = Vx + Z0 * Iy - V_max;
  V_(Vx_zmax, cx, cy, cz) = Vx - Z0 * Iy - V_min;
  V_min = V_(Vy_zmin, cx, cy, cz); V_max = V_(Vy_zmax, cx, cy, cz);
  V_(Vy_zmin, cx, cy, cz) = Vy - Z0 * Ix - V_max;
  V_(Vy_zmax, cx, cy, cz) = Vy + Z0 * Ix - V_min;
  V_min = V_(Vy_xmin, cx, cy, cz); V_max = V_(Vy_xmax, cx, cy, cz);
  V_(Vy_xmin, cx, cy, cz) = Vy + Z0 * Iz - V_max;
  V_(Vy_xmax, cx, cy, cz) = Vy - Z0 * Iz - V_min;
  V_min = V_(Vz_xmin, cx, cy, cz); V_max = V_(Vz_xmax, cx, cy, cz);
  V_(Vz_xmin, cx, cy, cz) = Vz - Z0 * Iy - V_max;
  V_(Vz_xmax, cx, cy, cz) = Vz + Z0 * Iy - V_min;
  V_min = V_(Vz_ymin, cx, cy, cz); V_max = V_(Vz_ymax, cx, cy, cz);
  V_(Vz_ymin, cx, cy, cz) = Vz + Z0 * Ix - V_max;
  V_(Vz_ymax, cx, cy, cz) = Vz - Z0 * Ix - V_min;
}

/* scatter(), TLM_SOLVER/scatter.F90:49-591, for the cells of plane cz; the
   output and excitation cell counters run on from *out_no / *exc_no */
static int scatter_plane(tlm_oracle_state *s, int cz, int *out_no, int *exc_no) {
  const tlm_oracle_problem *p = &s->p;
  const double dl = p->dl;
  const double Z04 = Z0 * 4.0, Y04 = Y0 * 4.0;
  int cell_number = (cz - 1) * s->ny * s->nx, output_cell_number = *out_no, excitation_cell_number = *exc_no;
  {
    for (int cy = 1; cy <= s->ny; cy++)
      for (int cx = 1; cx <= s->nx; cx++) {
        int code = p->cell_code[cell_number];
        cell_number++;
        if (code == 0) {
          /* free space, scatter.F90:222-272 */
          double Vx = (V_(Vx_ymin, cx, cy, cz) + V_(Vx_ymax, cx, cy, cz) + V_(Vx_zmin, cx, cy, cz) + V_(Vx_zmax, cx, cy, cz)) / 2.0;
          double Vy = (V_(Vy_xmin, cx, cy, cz) + V_(Vy_xmax, cx, cy, cz) + V_(Vy_zmin, cx, cy, cz) + V_(Vy_zmax, cx, cy, cz)) / 2.0;
          double Vz = (V_(Vz_xmin, cx, cy, cz) + V_(Vz_xmax, cx, cy, cz) + V_(Vz_ymin, cx, cy, cz) + V_(Vz_ymax, cx, cy, cz)) / 2.0;
          double Ix = (V_(Vz_ymax, cx, cy, cz) - V_(Vy_zmax, cx, cy, cz) - V_(Vz_ymin, cx, cy, cz) + V_(Vy_zmin, cx, cy, cz)) / (2.0 * Z0);
          double Iy = (V_(Vx_zmax, cx, cy, cz) - V_(Vz_xmax, cx, cy, cz) - V_(Vx_zmin, cx, cy, cz) + V_(Vz_xmin, cx, cy, cz)) / (2.0 * Z0);
          double Iz = (V_(Vy_xmax, cx, cy, cz) - V_(Vx_ymax, cx, cy, cz) - V_(Vy_xmin, cx, cy, cz) + V_(Vx_ymin, cx, cy, cz)) / (2.0 * Z0);
          scatter_pulses(s, cx, cy, cz, Vx, Vy, Vz, Ix, Iy, Iz);
          continue;
        }
        int sc = code - 1;
        int pml_cell = p->sp_pml[sc];
        int material_number = p->sp_material[sc];
        int material_type = material_number ? p->mat_type[material_number - 1] : 0;
        int output_number = p->sp_output[sc];
        if (pml_cell != 0) {
          if (material_type == 1 || material_type == 2) return -1; /* scatter.F90:559-567 */
          if (material_type == 3) { /* scatter.F90:570-571 */
            if (!p->pml_sigma) return -2;
            scatter_pml_material_cell(s, cx, cy, cz, pml_cell, material_number, output_number, &output_cell_number);
            continue;
          }
          scatter_pml_cell(s, cx, cy, cz, pml_cell, output_number, &output_cell_number);
          continue;
        }
        int excitation_number = p->sp_excitation[sc];
        int m = material_number - 1;
        /* scatter.F90:296-309 */
        double VEx = (V_(Vx_ymin, cx, cy, cz) + V_(Vx_ymax, cx, cy, cz) + V_(Vx_zmin, cx, cy, cz) + V_(Vx_zmax, cx, cy, cz)) / 2.0;
        double VEy = (V_(Vy_xmin, cx, cy, cz) + V_(Vy_xmax, cx, cy, cz) + V_(Vy_zmin, cx, cy, cz) + V_(Vy_zmax, cx, cy, cz)) / 2.0;
        double VEz = (V_(Vz_xmin, cx, cy, cz) + V_(Vz_xmax, cx, cy, cz) + V_(Vz_ymin, cx, cy, cz) + V_(Vz_ymax, cx, cy, cz)) / 2.0;
        double Yx = Y04, Yy = Y04, Yz = Y04;
        double VHx = 2.0 * (V_(Vz_ymax, cx, cy, cz) - V_(Vy_zmax, cx, cy, cz) - V_(Vz_ymin, cx, cy, cz) + V_(Vy_zmin, cx, cy, cz));
        double VHy = 2.0 * (V_(Vx_zmax, cx, cy, cz) - V_(Vz_xmax, cx, cy, cz) - V_(Vx_zmin, cx, cy, cz) + V_(Vz_xmin, cx, cy, cz));
        double VHz = 2.0 * (V_(Vy_xmax, cx, cy, cz) - V_(Vx_ymax, cx, cy, cz) - V_(Vy_xmin, cx, cy, cz) + V_(Vx_ymin, cx, cy, cz));
        double Zx = Z04, Zy = Z04, Zz = Z04;
        double Vox = 0, Voy = 0, Voz = 0, Ysx = 0, Ysy = 0, Ysz = 0;
        int filter_number = s->sp_filter[sc];
        const int MO = ORACLE_MAX_ORDER + 1;
        if (material_type == 1) {
          VEx = 0.0; VEy = 0.0; VEz = 0.0;
        } else if (material_type == 2) {
          VHx = 0.0; VHy = 0.0; VHz = 0.0;
        } else if (material_type == 3) {
          if (p->mat_eps_exists[m]) {
            Ysx = Ysy = Ysz = p->mat_Ys_eps_f[m];
            const double *a = p->mat_eps_a + (size_t)m * MO, *b = p->mat_eps_b + (size_t)m * MO;
            zresp_t *f0 = &s->eps_f[filter_number - 1];
            timeshift_Zfilter(&f0[0]); evaluate_Zfilter(a, b, &f0[0], 0.0); Vox = f0[0].f;
            timeshift_Zfilter(&f0[1]); evaluate_Zfilter(a, b, &f0[1], 0.0); Voy = f0[1].f;
            timeshift_Zfilter(&f0[2]); evaluate_Zfilter(a, b, &f0[2], 0.0); Voz = f0[2].f;
            add_shunt_admittance(&VEx, &Yx, Vox, Ysx);
            add_shunt_admittance(&VEy, &Yy, Voy, Ysy);
            add_shunt_admittance(&VEz, &Yz, Voz, Ysz);
          }
          double Ge = p->mat_Ge[m];
          add_shunt_admittance(&VEx, &Yx, 0.0, Ge);
          add_shunt_admittance(&VEy, &Yy, 0.0, Ge);
          add_shunt_admittance(&VEz, &Yz, 0.0, Ge);
          if (p->mat_mu_exists[m]) {
            double Zs = p->mat_Zs_mu_f[m];
            const double *a = p->mat_mu_a + (size_t)m * MO, *b = p->mat_mu_b + (size_t)m * MO;
            zresp_t *f0 = &s->mu_f[filter_number - 1];
            double Vsx, Vsy, Vsz;
            timeshift_Zfilter(&f0[0]); evaluate_Zfilter(a, b, &f0[0], 0.0); Vsx = f0[0].f;
            timeshift_Zfilter(&f0[1]); evaluate_Zfilter(a, b, &f0[1], 0.0); Vsy = f0[1].f;
            timeshift_Zfilter(&f0[2]); evaluate_Zfilter(a, b, &f0[2], 0.0); Vsz = f0[2].f;
            add_series_impedance(&VHx, &Zx, Vsx, Zs);
            add_series_impedance(&VHy, &Zy, Vsy, Zs);
            add_series_impedance(&VHz, &Zz, Vsz, Zs);
          }
          double Rm = p->mat_Rm[m];
          add_series_impedance(&VHx, &Zx, 0.0, Rm);
          add_series_impedance(&VHy, &Zy, 0.0, Rm);
          add_series_impedance(&VHz, &Zz, 0.0, Rm);
        }
        double Vx = VEx, Vy = VEy, Vz = VEz;
        double Ix = VHx / Zx, Iy = VHy / Zy, Iz = VHz / Zz;
        if (excitation_number != 0) {
          /* scatter.F90:429-450 */
          const double *field = s->cell_exc + (size_t)excitation_cell_number * 9;
          const int32_t *h = s->cell_exc_type + (size_t)excitation_cell_number * 6;
          excitation_cell_number++;
          double Isx = field[Jx] * dl * dl, Isy = field[Jy] * dl * dl, Isz = field[Jz] * dl * dl;
          Vx = (double)h[0] * Vx - field[Ex] * dl / 2.0 + Isx / Yx;
          Vy = (double)h[1] * Vy - field[Ey] * dl / 2.0 + Isy / Yy;
          Vz = (double)h[2] * Vz - field[Ez] * dl / 2.0 + Isz / Yz;
          Ix = (double)h[3] * Ix + field[Hx] * dl / 2.0;
          Iy = (double)h[4] * Iy + field[Hy] * dl / 2.0;
          Iz = (double)h[5] * Iz + field[Hz] * dl / 2.0;
        }
        if (output_number != 0) {
          /* scatter.F90:465-480 */
          double *f = s->cell_out + (size_t)output_cell_number * 6;
          output_cell_number++;
          f[Ex] = -Vx / dl; f[Ey] = -Vy / dl; f[Ez] = -Vz / dl;
          f[Hx] = Ix / dl; f[Hy] = Iy / dl; f[Hz] = Iz / dl;
        }
        if (material_type == 3) {
          /* scatter.F90:483-515 */
          if (p->mat_eps_exists[m]) {
            const double *a = p->mat_eps_a + (size_t)m * MO, *b = p->mat_eps_b + (size_t)m * MO;
            zresp_t *f0 = &s->eps_f[filter_number - 1];
            double Iox = (Vx - Vox) * Ysx, Ioy = (Vy - Voy) * Ysy, Ioz = (Vz - Voz) * Ysz;
            evaluate_Zfilter(a, b, &f0[0], Iox);
            evaluate_Zfilter(a, b, &f0[1], Ioy);
            evaluate_Zfilter(a, b, &f0[2], Ioz);
          }
          if (p->mat_mu_exists[m]) {
            const double *a = p->mat_mu_a + (size_t)m * MO, *b = p->mat_mu_b + (size_t)m * MO;
            zresp_t *f0 = &s->mu_f[filter_number - 1];
            evaluate_Zfilter(a, b, &f0[0], -Ix);
            evaluate_Zfilter(a, b, &f0[1], -Iy);
            evaluate_Zfilter(a, b, &f0[2], -Iz);
          }
        }
        scatter_pulses(s, cx, cy, cz, Vx, Vy, Vz, Ix, Iy, Iz);
      }
  }
  *out_no = output_cell_number;
  *exc_no = excitation_cell_number;
  return 0;
}

static void connect_plane(tlm_oracle_state *s, int cz, int excitation_face_number, int output_face_number);

/* z-planes shared among s->threads POSIX threads in contiguous slabs, each
   plane starting from the counters of the sequential traversal */
typedef struct {
  tlm_oracle_state *s;
  int pass, z0, z1, rc;
} plane_job;

static void *plane_worker(void *arg) {
  plane_job *j = (plane_job *)arg;
  tlm_oracle_state *s = j->s;
  for (int cz = j->z0; cz <= j->z1; cz++) {
    if (j->pass == 0) {
      int out_no = s->plane_out0[cz - 1], exc_no = s->plane_exc0[cz - 1];
      int rc = scatter_plane(s, cz, &out_no, &exc_no);
      if (rc && !j->rc) j->rc = rc;
    } else {
      connect_plane(s, cz, s->plane_fexc0[cz - 1], s->plane_fout0[cz - 1]);
    }
  }
  return NULL;
}

static int run_planes(tlm_oracle_state *s, int pass) {
  int T = s->threads < s->nz ? s->threads : s->nz;
  if (T > 256) T = 256;
  plane_job jobs[256];
  pthread_t th[256];
  int started[256];
  for (int t = 0; t < T; t++) {
    jobs[t].s = s;
    jobs[t].pass = pass;
    jobs[t].z0 = 1 + (int)((long long)s->nz * t / T);
    jobs[t].z1 = (int)((long long)s->nz * (t + 1) / T);
    jobs[t].rc = 0;
    started[t] = t > 0 && pthread_create(&th[t], NULL, plane_worker, &jobs[t]) == 0;
    if (t > 0 && !started[t]) plane_worker(&jobs[t]); /* no thread: do the slab here */
  }
  plane_worker(&jobs[0]);
  int rc = 0;
  for (int t = 0; t < T; t++) {
    if (t > 0 && started[t]) pthread_join(th[t], NULL);
    if (jobs[t].rc && !rc) rc = jobs[t].rc;
  }
  return rc;
}

/* scatter() over all planes: in traversal order on one thread, or planes
   shared among threads with the counters each plane starts from */
static int scatter(tlm_oracle_state *s) {
  if (s->threads <= 1) {
    int out_no = 0, exc_no = 0;
    for (int cz = 1; cz <= s->nz; cz++) {
      int rc = scatter_plane(s, cz, &out_no, &exc_no);
      if (rc) return rc;
    }
    return 0;
  }
  return run_planes(s, 0);
}

/* surface_material_update (MATERIALS/TLM_surface_materials.F90:535-697):
   a thin layer as a two-port impedance matrix between the incident pulses
   from the left (the cell below the face) and the right; both sides see
   the line impedance Z0.  flt: the four filter responses Z11, Z12, Z21, Z22
   of this face and polarisation.  Returns -3 when the matrix is singular
   (the reference stops there). */
static int thin_layer_update(const tlm_oracle_problem *p, int m, int pol, int reverse, zresp_t *flt, double Vli,
                             double Vri, double *Vl, double *Vr) {
  const int MO = ORACLE_MAX_ORDER + 1, base = (m * 3 + pol) * 4;
  const double *f = p->smat_f + base;
  double slow[4];
  for (int k = 0; k < 4; k++) {
    evaluate_Zfilter(p->smat_a + (size_t)(base + k) * MO, p->smat_b + (size_t)(base + k) * MO, &flt[k], 0.0);
    slow[k] = flt[k].f;
  }
  double Zl = Z0, Zr = Z0;
  double Z1 = reverse ? Zr : Zl, Z2 = reverse ? Zl : Zr;
  double U11 = Z1 + f[0], U12 = f[1], U21 = f[2], U22 = Z2 + f[3];
  double det = U11 * U22 - U21 * U12;
  if (det == 0.0) return -3;
  double V1i = reverse ? Vri : Vli, V2i = reverse ? Vli : Vri;
  double rhs1 = 2.0 * V1i - slow[0] - slow[1];
  double rhs2 = 2.0 * V2i - slow[2] - slow[3];
  double i1 = (U22 * rhs1 - U12 * rhs2) / det;
  double i2 = (-U21 * rhs1 + U11 * rhs2) / det;
  double V1 = 2.0 * V1i - i1 * Z1;
  double V2 = 2.0 * V2i - i2 * Z2;
  const double G[4] = {i1, i2, i1, i2};
  for (int k = 0; k < 4; k++)
    evaluate_Zfilter(p->smat_a + (size_t)(base + k) * MO, p->smat_b + (size_t)(base + k) * MO, &flt[k], G[k]);
  *Vl = reverse ? V2 : V1;
  *Vr = reverse ? V1 : V2;
  for (int k = 0; k < 4; k++) timeshift_Zfilter(&flt[k]);
  return 0;
}

/* one special face of connect(): connect_normal_to_{x,y,z}.F90 for faces
   with no surface material (material_type 0), face excitation and face output.
   pa/pb are the two port pairs (min port on cell c, max port on cell c-1). */
static void connect_special_face(tlm_oracle_state *s, int f, int cx, int cy, int cz, int dir,
                                 int *excitation_face_number, int *output_face_number) {
  const tlm_oracle_problem *p = &s->p;
  const double dl = p->dl;
  int mx = cx, my = cy, mz = cz; /* cell on the min side of the face */
  int pmin1, pmax1, pmin2, pmax2;
  if (dir == 1) { mx = cx - 1; pmin1 = Vy_xmin; pmax1 = Vy_xmax; pmin2 = Vz_xmin; pmax2 = Vz_xmax; }
  else if (dir == 2) { my = cy - 1; pmin1 = Vx_ymin; pmax1 = Vx_ymax; pmin2 = Vz_ymin; pmax2 = Vz_ymax; }
  else { mz = cz - 1; pmin1 = Vx_zmin; pmax1 = Vx_zmax; pmin2 = Vy_zmin; pmax2 = Vy_zmax; }
  int out = p->face_out[f], exc = p->face_exc[f];
  /* incident (before connect) pulses for output: *_negative_1, *_positive_2 */
  double n1a = V_(pmin1, cx, cy, cz), n1b = V_(pmin2, cx, cy, cz);
  double p2a = V_(pmax1, mx, my, mz), p2b = V_(pmax2, mx, my, mz);
  double A_min = V_(pmin1, cx, cy, cz) + V_(pmax1, mx, my, mz), A_max = A_min;
  double B_min = V_(pmin2, cx, cy, cz) + V_(pmax2, mx, my, mz), B_max = B_min;
  const int mat = p->face_mat ? p->face_mat[f] : 0;
  if (mat == 1) { /* PEC sheet: connect_normal_to_x.F90:36-40 */
    A_min = 0.0; A_max = 0.0; B_min = 0.0; B_max = 0.0;
  } else if (mat == 2) { /* PMC sheet: connect_normal_to_x.F90:41-45 */
    A_min = 2.0 * V_(pmin1, cx, cy, cz); A_max = 2.0 * V_(pmax1, mx, my, mz);
    B_min = 2.0 * V_(pmin2, cx, cy, cz); B_max = 2.0 * V_(pmax2, mx, my, mz);
  } else if (mat == 3) { /* thin layer: connect_normal_to_x.F90:268-282 (y, z analogues) */
    int sm = p->face_smat[f], m = abs(sm) - 1;
    int pol1 = dir == 1 ? 1 : 0, pol2 = dir == 3 ? 1 : 2;
    zresp_t *flt = s->sm_f + (size_t)f * 8;
    int rc = thin_layer_update(p, m, pol1, sm > 0, flt, V_(pmax1, mx, my, mz), V_(pmin1, cx, cy, cz), &A_max, &A_min);
    if (!rc) rc = thin_layer_update(p, m, pol2, sm > 0, flt + 4, V_(pmax2, mx, my, mz), V_(pmin2, cx, cy, cz),
                                    &B_max, &B_min);
    if (rc) s->err = rc;
  } /* 0 and 4 (free-space surface material): the plain sum */
  if (exc != 0) {
    const double *fmin = s->face_exc + (size_t)(*excitation_face_number) * 24;
    const double *fmax = fmin + 12;
    const int32_t *hmin = s->face_exc_type + (size_t)(*excitation_face_number) * 12;
    const int32_t *hmax = hmin; /* side-1 types on both sides, connect_normal_to_x.F90:293-294 */
    (*excitation_face_number)++;
    const double *Jsn = fmin + Jx, *Jsx_ = fmax + Jx, *Msn = fmin + Mx, *Msx_ = fmax + Mx;
    if (dir == 1) { /* connect_normal_to_x.F90:301-305 */
      A_min = A_min * hmin[Ey] - fmin[Ey] * dl - fmin[Hz] * Z0 * dl + Jsn[1] * dl * Z0 / 2.0 + Msn[2] * dl / 2.0;
      A_max = A_max * hmax[Ey] - fmax[Ey] * dl + fmax[Hz] * Z0 * dl + Jsx_[1] * dl * Z0 / 2.0 - Msx_[2] * dl / 2.0;
      B_min = B_min * hmin[Ez] - fmin[Ez] * dl + fmin[Hy] * Z0 * dl + Jsn[2] * dl * Z0 / 2.0 - Msn[1] * dl / 2.0;
      B_max = B_max * hmax[Ez] - fmax[Ez] * dl - fmax[Hy] * Z0 * dl + Jsx_[2] * dl * Z0 / 2.0 + Msx_[1] * dl / 2.0;
    } else if (dir == 2) { /* connect_normal_to_y.F90:304-308 */
      A_min = A_min * hmin[Ex] - fmin[Ex] * dl + fmin[Hz] * Z0 * dl + Jsn[0] * dl * Z0 / 2.0 - Msn[2] * dl / 2.0;
      A_max = A_max * hmax[Ex] - fmax[Ex] * dl - fmax[Hz] * Z0 * dl + Jsx_[0] * dl * Z0 / 2.0 + Msx_[2] * dl / 2.0;
      B_min = B_min * hmin[Ez] - fmin[Ez] * dl - fmin[Hx] * Z0 * dl + Jsn[2] * dl * Z0 / 2.0 + Msn[0] * dl / 2.0;
      B_max = B_max * hmax[Ez] - fmax[Ez] * dl + fmax[Hx] * Z0 * dl + Jsx_[2] * dl * Z0 / 2.0 - Msx_[0] * dl / 2.0;
    } else { /* connect_normal_to_z.F90:302-306 */
      A_min = A_min * hmin[Ex] - fmin[Ex] * dl - fmin[Hy] * Z0 * dl + Jsn[0] * dl * Z0 / 2.0 + Msn[1] * dl / 2.0;
      A_max = A_max * hmax[Ex] - fmax[Ex] * dl + fmax[Hy] * Z0 * dl + Jsx_[0] * dl * Z0 / 2.0 - Msx_[1] * dl / 2.0;
      B_min = B_min * hmin[Ey] - fmin[Ey] * dl + fmin[Hx] * Z0 * dl + Jsn[1] * dl * Z0 / 2.0 - Msn[0] * dl / 2.0;
      B_max = B_max * hmax[Ey] - fmax[Ey] * dl - fmax[Hx] * Z0 * dl + Jsx_[1] * dl * Z0 / 2.0 + Msx_[0] * dl / 2.0;
    }
  }
  V_(pmax1, mx, my, mz) = A_max - V_(pmax1, mx, my, mz);
  V_(pmin1, cx, cy, cz) = A_min - V_(pmin1, cx, cy, cz);
  V_(pmax2, mx, my, mz) = B_max - V_(pmax2, mx, my, mz);
  V_(pmin2, cx, cy, cz) = B_min - V_(pmin2, cx, cy, cz);
  if (out != 0) {
    double p1a = V_(pmin1, cx, cy, cz), p1b = V_(pmin2, cx, cy, cz);
    double n2a = V_(pmax1, mx, my, mz), n2b = V_(pmax2, mx, my, mz);
    double *fo = s->face_out + (size_t)(*output_face_number) * 12;
    (*output_face_number)++;
    for (int side = 0; side < 2; side++) {
      double pa = side ? p2a : p1a, na = side ? n2a : n1a;
      double pb = side ? p2b : p1b, nb = side ? n2b : n1b;
      double *fld = fo + side * 6;
      if (dir == 1) { /* connect_normal_to_x.F90:334-352 */
        fld[Ex] = 0.0; fld[Ey] = -(pa + na) / dl; fld[Ez] = -(pb + nb) / dl;
        fld[Hx] = 0.0; fld[Hy] = (pb - nb) / (Z0 * dl); fld[Hz] = -(pa - na) / (Z0 * dl);
      } else if (dir == 2) { /* connect_normal_to_y.F90 output */
        fld[Ex] = -(pa + na) / dl; fld[Ey] = 0.0; fld[Ez] = -(pb + nb) / dl;
        fld[Hx] = -(pb - nb) / (Z0 * dl); fld[Hy] = 0.0; fld[Hz] = (pa - na) / (Z0 * dl);
      } else { /* connect_normal_to_z.F90:338-360 */
        fld[Ex] = -(pa + na) / dl; fld[Ey] = -(pb + nb) / dl; fld[Ez] = 0.0;
        fld[Hx] = (pb - nb) / (Z0 * dl); fld[Hy] = -(pa - na) / (Z0 * dl); fld[Hz] = 0.0;
      }
    }
  }
}

/* connect(), TLM_SOLVER/connect.F90:180-214 with the free-space branches of
   connect_normal_to_{x,y,z}.F90:1-10 */
static void connect_plane(tlm_oracle_state *s, int cz, int excitation_face_number, int output_face_number) {
  size_t cell = (size_t)(cz - 1) * s->ny * s->nx;
  {
    for (int cy = 1; cy <= s->ny; cy++)
      for (int cx = 1; cx <= s->nx; cx++, cell++) {
        if (cx != 1) {
          int f = s->face_code[cell * 3 + 0];
          if (f == 0) {
            double Vy = V_(Vy_xmin, cx, cy, cz) + V_(Vy_xmax, cx - 1, cy, cz);
            V_(Vy_xmin, cx, cy, cz) = Vy - V_(Vy_xmin, cx, cy, cz);
            V_(Vy_xmax, cx - 1, cy, cz) = Vy - V_(Vy_xmax, cx - 1, cy, cz);
            double Vz = V_(Vz_xmin, cx, cy, cz) + V_(Vz_xmax, cx - 1, cy, cz);
            V_(Vz_xmin, cx, cy, cz) = Vz - V_(Vz_xmin, cx, cy, cz);
            V_(Vz_xmax, cx - 1, cy, cz) = Vz - V_(Vz_xmax, cx - 1, cy, cz);
          } else {
            connect_special_face(s, f - 1, cx, cy, cz, 1, &excitation_face_number, &output_face_number);
          }
        }
        if (cy != 1) {
          int f = s->face_code[cell * 3 + 1];
          if (f == 0) {
            double Vx = V_(Vx_ymin, cx, cy, cz) + V_(Vx_ymax, cx, cy - 1, cz);
            V_(Vx_ymin, cx, cy, cz) = Vx - V_(Vx_ymin, cx, cy, cz);
            V_(Vx_ymax, cx, cy - 1, cz) = Vx - V_(Vx_ymax, cx, cy - 1, cz);
            double Vz = V_(Vz_ymin, cx, cy, cz) + V_(Vz_ymax, cx, cy - 1, cz);
            V_(Vz_ymin, cx, cy, cz) = Vz - V_(Vz_ymin, cx, cy, cz);
            V_(Vz_ymax, cx, cy - 1, cz) = Vz - V_(Vz_ymax, cx, cy - 1, cz);
          } else {
            connect_special_face(s, f - 1, cx, cy, cz, 2, &excitation_face_number, &output_face_number);
          }
        }
        if (cz != 1 || s->p.slab[0]) {  /* the z-face below a slab's first plane: connected here */
          int f = cz != 1 ? s->face_code[cell * 3 + 2] : 0;
          if (f == 0) {
            double Vx = V_(Vx_zmin, cx, cy, cz) + V_(Vx_zmax, cx, cy, cz - 1);
            V_(Vx_zmin, cx, cy, cz) = Vx - V_(Vx_zmin, cx, cy, cz);
            V_(Vx_zmax, cx, cy, cz - 1) = Vx - V_(Vx_zmax, cx, cy, cz - 1);
            double Vy = V_(Vy_zmin, cx, cy, cz) + V_(Vy_zmax, cx, cy, cz - 1);
            V_(Vy_zmin, cx, cy, cz) = Vy - V_(Vy_zmin, cx, cy, cz);
            V_(Vy_zmax, cx, cy, cz - 1) = Vy - V_(Vy_zmax, cx, cy, cz - 1);
          } else {
            connect_special_face(s, f - 1, cx, cy, cz, 3, &excitation_face_number, &output_face_number);
          }
        }
      }
  }
}

/* Every port takes part in exactly one face, so the faces of different
   planes touch disjoint ports and the planes can be connected in any order
   or at once, with the same result. */
static void connect(tlm_oracle_state *s) {
  if (s->threads <= 1) {
    for (int cz = 1; cz <= s->nz; cz++) connect_plane(s, cz, s->plane_fexc0[cz - 1], s->plane_fout0[cz - 1]);
    return;
  }
  run_planes(s, 1);
}

/* outer_boundary(), TLM_SOLVER/outer_boundary.F90:71-131 */
static void outer_boundary(tlm_oracle_state *s, int timestep) {
  const double *R = s->p.R;
  const tlm_oracle_problem *p = &s->p;
  int nx = s->nx, ny = s->ny, nz = s->nz;
  for (int cz = 1; cz <= nz; cz++)
    for (int cy = 1; cy <= ny; cy++) {
      V_(Vy_xmin, 1, cy, cz) = V_(Vy_xmin, 1, cy, cz) * R[0];
      V_(Vz_xmin, 1, cy, cz) = V_(Vz_xmin, 1, cy, cz) * R[0];
      V_(Vy_xmax, nx, cy, cz) = V_(Vy_xmax, nx, cy, cz) * R[1];
      V_(Vz_xmax, nx, cy, cz) = V_(Vz_xmax, nx, cy, cz) * R[1];
    }
  for (int cz = 1; cz <= nz; cz++)
    for (int cx = 1; cx <= nx; cx++) {
      V_(Vx_ymin, cx, 1, cz) = V_(Vx_ymin, cx, 1, cz) * R[2];
      V_(Vz_ymin, cx, 1, cz) = V_(Vz_ymin, cx, 1, cz) * R[2];
      V_(Vx_ymax, cx, ny, cz) = V_(Vx_ymax, cx, ny, cz) * R[3];
      V_(Vz_ymax, cx, ny, cz) = V_(Vz_ymax, cx, ny, cz) * R[3];
    }
  if (!p->slab[0])
    for (int cy = 1; cy <= ny; cy++)
      for (int cx = 1; cx <= nx; cx++) {
        V_(Vx_zmin, cx, cy, 1) = V_(Vx_zmin, cx, cy, 1) * R[4];
        V_(Vy_zmin, cx, cy, 1) = V_(Vy_zmin, cx, cy, 1) * R[4];
      }
  if (!p->slab[1])
    for (int cy = 1; cy <= ny; cy++)
      for (int cx = 1; cx <= nx; cx++) {
        V_(Vx_zmax, cx, cy, nz) = V_(Vx_zmax, cx, cy, nz) * R[5];
        V_(Vy_zmax, cx, cy, nz) = V_(Vy_zmax, cx, cy, nz) * R[5];
      }
  if (!p->hs_outer) return;
  /* outer-boundary Huygens surface (outer_boundary.F90:133-318): per
     boundary face, the two tangential ports get
     V - J dl Z0/2 + sg M dl/2 + R (-J dl Z0/2 - sg M dl/2)
     with (port, J component, M component, sg) per face code below */
  static const int tab[7][2][4] = {
      {{0}},
      {{Vy_xmin, 1, 2, -1}, {Vz_xmin, 2, 1, +1}}, /* face_xmin */
      {{Vx_ymin, 0, 2, +1}, {Vz_ymin, 2, 0, -1}}, /* face_ymin */
      {{Vx_zmin, 0, 1, -1}, {Vy_zmin, 1, 0, +1}}, /* face_zmin */
      {{Vy_xmax, 1, 2, +1}, {Vz_xmax, 2, 1, -1}}, /* face_xmax */
      {{Vx_ymax, 0, 2, -1}, {Vz_ymax, 2, 0, +1}}, /* face_ymax */
      {{Vx_zmax, 0, 1, +1}, {Vy_zmax, 1, 0, -1}}, /* face_zmax */
  };
  const double dl = p->dl;
  for (int h = 0; h < p->hs_n; h++) {
    const int32_t *c = p->hs_cell + 4 * h;
    double value = interp_face_value(s, p->hs_offset[h], timestep);
    double normx = p->hs_norm[3 * h], normy = p->hs_norm[3 * h + 1], normz = p->hs_norm[3 * h + 2];
    const double *Hi = p->hs_Hi, *Ei = p->hs_Ei;
    double Js[3], Ms[3];
    Js[0] = (normy * value * (Hi[2]) - normz * value * (Hi[1]));
    Js[1] = (normz * value * (Hi[0]) - normx * value * (Hi[2]));
    Js[2] = (normx * value * (Hi[1]) - normy * value * (Hi[0]));
    Ms[0] = -(normy * value * (Ei[2]) - normz * value * (Ei[1]));
    Ms[1] = -(normz * value * (Ei[0]) - normx * value * (Ei[2]));
    Ms[2] = -(normx * value * (Ei[1]) - normy * value * (Ei[0]));
    const int code = c[3];
    const double Rf = R[code <= 3 ? 2 * (code - 1) : 2 * (code - 4) + 1];
    for (int q = 0; q < 2; q++) {
      const int port = tab[code][q][0];
      const double J = Js[tab[code][q][1]], M = Ms[tab[code][q][2]], sg = tab[code][q][3];
      double *v = &V_(port, c[0], c[1], c[2]);
      *v = *v - J * dl * Z0 / 2.0 + sg * M * dl / 2.0 + Rf * (-J * dl * Z0 / 2.0 - sg * M * dl / 2.0);
    }
  }
}

/* wrap_outer_boundary, TLM_SOLVER/wrap_outer_boundary.F90:101-273 (one
   process): the ports of the two outer faces of a wrapped axis swap */
static void wrap_outer_boundary(tlm_oracle_state *s) {
  const tlm_oracle_problem *p = &s->p;
  int nx = s->nx, ny = s->ny, nz = s->nz;
  if (p->wrap[0])
    for (int cz = 1; cz <= nz; cz++)
      for (int cy = 1; cy <= ny; cy++) {
        double Vy = V_(Vy_xmin, 1, cy, cz);
        V_(Vy_xmin, 1, cy, cz) = V_(Vy_xmax, nx, cy, cz);
        V_(Vy_xmax, nx, cy, cz) = Vy;
        double Vz = V_(Vz_xmin, 1, cy, cz);
        V_(Vz_xmin, 1, cy, cz) = V_(Vz_xmax, nx, cy, cz);
        V_(Vz_xmax, nx, cy, cz) = Vz;
      }
  if (p->wrap[1])
    for (int cz = 1; cz <= nz; cz++)
      for (int cx = 1; cx <= nx; cx++) {
        double Vx = V_(Vx_ymin, cx, 1, cz);
        V_(Vx_ymin, cx, 1, cz) = V_(Vx_ymax, cx, ny, cz);
        V_(Vx_ymax, cx, ny, cz) = Vx;
        double Vz = V_(Vz_ymin, cx, 1, cz);
        V_(Vz_ymin, cx, 1, cz) = V_(Vz_ymax, cx, ny, cz);
        V_(Vz_ymax, cx, ny, cz) = Vz;
      }
  if (p->wrap[2])
    for (int cy = 1; cy <= ny; cy++)
      for (int cx = 1; cx <= nx; cx++) {
        double Vx = V_(Vx_zmin, cx, cy, 1);
        V_(Vx_zmin, cx, cy, 1) = V_(Vx_zmax, cx, cy, nz);
        V_(Vx_zmax, cx, cy, nz) = Vx;
        double Vy = V_(Vy_zmin, cx, cy, 1);
        V_(Vy_zmin, cx, cy, 1) = V_(Vy_zmax, cx, cy, nz);
        V_(Vy_zmax, cx, cy, nz) = Vy;
      }
}

/* face_output_frequency_output_surfaces, frequency_output_surfaces.F90:297-421 */
/* get_output_flag, OUTPUT/output.F90:564-598 */
static int output_flag(int timestep, int first, int last, int interval) {
  if (timestep < first || timestep > last) return 0;
  return (timestep - first) % interval == 0;
}

static void dft_surfaces(tlm_oracle_state *s, double time, int timestep) {
  const tlm_oracle_problem *p = &s->p;
  const double pi = 3.141592653589793;
  for (int d = 0; d < p->n_dft; d++) {
    if (p->dft_gate && !output_flag(timestep, p->dft_gate[3 * d], p->dft_gate[3 * d + 1], p->dft_gate[3 * d + 2]))
      continue;
    double arg = -2.0 * pi * p->dft_freq[d] * time;
    double er = cos(arg), ei = sin(arg); /* exp(-j*2*pi*f*t) */
    int comp = p->dft_comp[d];
    for (int k = p->dft_face_ptr[d]; k < p->dft_face_ptr[d + 1]; k++) {
      int face = p->dft_face_side[k];
      int side = (face <= 3) ? 0 : 1;
      double normx = 0, normy = 0, normz = 0;
      if (face == 1) normx = 1; else if (face == 4) normx = -1;
      else if (face == 2) normy = 1; else if (face == 5) normy = -1;
      else if (face == 3) normz = 1; else normz = -1;
      const double *fld = s->face_out + (size_t)(p->dft_face_out[k] - 1) * 12 + side * 6;
      double value;
      if (comp <= 6) value = fld[comp - 1];
      else if (comp == 7) value = (normy * fld[Hz] - normz * fld[Hy]);
      else if (comp == 8) value = (normz * fld[Hx] - normx * fld[Hz]);
      else value = (normx * fld[Hy] - normy * fld[Hx]);
      s->dft[2 * k] = s->dft[2 * k] + value * er;
      s->dft[2 * k + 1] = s->dft[2 * k + 1] + value * ei;
    }
  }
}

/* face_output_far_field, far_field_surfaces.F90:252-351: J += e^{-jwt} dt (n x H),
   M -= e^{-jwt} dt (n x E) on the face side of each entry, n = +1 on a min
   face and -1 on a max face */
static void far_field_surfaces(tlm_oracle_state *s, double time) {
  const tlm_oracle_problem *p = &s->p;
  const double pi = 3.141592653589793;
  for (int d = 0; d < p->n_ff; d++) {
    double arg = -2.0 * pi * p->ff_freq[d] * time;
    double er = cos(arg) * p->dt, ei = sin(arg) * p->dt; /* exp(-j*2*pi*f*t)*dt */
    for (int k = p->ff_face_ptr[d]; k < p->ff_face_ptr[d + 1]; k++) {
      int face = p->ff_face_code[k];
      int side = (face <= 3) ? 0 : 1;
      double normx = 0, normy = 0, normz = 0;
      if (face == 1) normx = 1; else if (face == 4) normx = -1;
      else if (face == 2) normy = 1; else if (face == 5) normy = -1;
      else if (face == 3) normz = 1; else normz = -1;
      const double *fld = s->face_out + (size_t)(p->ff_face_out[k] - 1) * 12 + side * 6;
      double v[6];
      v[0] = (normy * fld[Hz] - normz * fld[Hy]);
      v[1] = (normz * fld[Hx] - normx * fld[Hz]);
      v[2] = (normx * fld[Hy] - normy * fld[Hx]);
      v[3] = (normy * fld[Ez] - normz * fld[Ey]);
      v[4] = (normz * fld[Ex] - normx * fld[Ez]);
      v[5] = (normx * fld[Ey] - normy * fld[Ex]);
      double *a = s->ff_acc + (size_t)k * 12;
      for (int c = 0; c < 3; c++) {
        a[2 * c] = a[2 * c] + er * v[c];
        a[2 * c + 1] = a[2 * c + 1] + ei * v[c];
        a[6 + 2 * c] = a[6 + 2 * c] - er * v[3 + c];
        a[6 + 2 * c + 1] = a[6 + 2 * c + 1] - ei * v[3 + c];
      }
    }
  }
}

/* run_TLM.F90:191-295 for timesteps first..first+n-1 */
/* TLM_set_small_to_zero (TLM_SOLVER/TLM_set_small_to_zero.F90:34-68): the 12
   incident pulses of every cell with |V| below the threshold become 0 */
static void set_small_to_zero(tlm_oracle_state *s) {
  const double small = s->p.small_to_zero_value;
  for (int cz = 1; cz <= s->nz; cz++)
    for (int cy = 1; cy <= s->ny; cy++)
      for (int cx = 1; cx <= s->nx; cx++)
        for (int port = 0; port < 12; port++)
          if (fabs(V_(port, cx, cy, cz)) < small) V_(port, cx, cy, cz) = 0.0;
}

int tlm_oracle_half_step(tlm_oracle_state *s, int32_t timestep, int32_t half, double *cell_out) {
  const tlm_oracle_problem *p = &s->p;
  if (timestep != s->timestep + 1) return -10;
  if (half == 1) {
    /* run_TLM.F90:236-238, before the excitation of the step */
    if (p->n_small_to_zero > 0 && timestep % p->n_small_to_zero == 0) set_small_to_zero(s);
    excitation(s, timestep);
    int rc = scatter(s);
    if (rc) return rc;
    if (cell_out && p->n_out_cells) memcpy(cell_out, s->cell_out, sizeof(double) * p->n_out_cells * 6);
    return 0;
  }
  if (half != 2) return -11;
  double time = (timestep - 1) * p->dt + p->dt / 2.0;
  connect(s);
  if (s->err) return s->err;
  /* face_output_points (output_points.F90:255-444): side 1/2 of the output face */
  for (int q = 0; q < p->n_face_probes; q++)
    s->face_probe_rec[(size_t)(timestep - 1) * p->n_face_probes + q] =
        s->face_out[(size_t)(p->fprobe_face[q] - 1) * 12 + (p->fprobe_side[q] - 1) * 6 + (p->fprobe_comp[q] - 1)];
  dft_surfaces(s, time, timestep);
  far_field_surfaces(s, time);
  outer_boundary(s, timestep);
  wrap_outer_boundary(s);
  s->timestep = timestep;
  return 0;
}

int tlm_oracle_run(tlm_oracle_state *s, int32_t first_step, int32_t n_steps, double *cell_out) {
  const tlm_oracle_problem *p = &s->p;
  if (first_step != s->timestep + 1) return -10;
  for (int k = 0; k < n_steps; k++) {
    int rc = tlm_oracle_half_step(s, first_step + k, 1, cell_out ? cell_out + (size_t)k * p->n_out_cells * 6 : NULL);
    if (rc) return rc;
    rc = tlm_oracle_half_step(s, first_step + k, 2, NULL);
    if (rc) return rc;
  }
  return 0;
}

int tlm_oracle_get_zplane(tlm_oracle_state *s, int32_t plane, double *out) {
  if (plane != 0 && plane != 1) return -11;
  const int cz = plane ? s->nz : 0;
  size_t k = 0;
  for (int port = 0; port < 2; port++)
    for (int cy = 1; cy <= s->ny; cy++)
      for (int cx = 1; cx <= s->nx; cx++) out[k++] = V_(port ? Vy_zmax : Vx_zmax, cx, cy, cz);
  return 0;
}

int tlm_oracle_set_zplane(tlm_oracle_state *s, int32_t plane, const double *in) {
  if (plane != 0 && plane != 1) return -11;
  const int cz = plane ? s->nz : 0;
  size_t k = 0;
  for (int port = 0; port < 2; port++)
    for (int cy = 1; cy <= s->ny; cy++)
      for (int cx = 1; cx <= s->nx; cx++) V_(port ? Vy_zmax : Vx_zmax, cx, cy, cz) = in[k++];
  return 0;
}

int tlm_oracle_get_dft(tlm_oracle_state *s, double *out) {
  int n = s->p.n_dft ? s->p.dft_face_ptr[s->p.n_dft] : 0;
  memcpy(out, s->dft, sizeof(double) * 2 * (size_t)n);
  return 0;
}

int tlm_oracle_get_far_field(tlm_oracle_state *s, double *out) {
  memcpy(out, s->ff_acc, sizeof(double) * 12 * (size_t)(s->p.n_ff ? s->p.ff_face_ptr[s->p.n_ff] : 0));
  return 0;
}

int tlm_oracle_get_face_probes(tlm_oracle_state *s, double *out) {
  memcpy(out, s->face_probe_rec, sizeof(double) * (size_t)s->timestep * s->p.n_face_probes);
  return 0;
}

int tlm_oracle_get_links(tlm_oracle_state *s, double *out) {
  size_t i = 0;
  for (int cz = 1; cz <= s->nz; cz++)
    for (int cy = 1; cy <= s->ny; cy++)
      for (int cx = 1; cx <= s->nx; cx++)
        for (int port = 0; port < 12; port++) out[i++] = V_(port, cx, cy, cz);
  return 0;
}

int tlm_oracle_set_threads(tlm_oracle_state *s, int32_t threads) {
  s->threads = threads < 1 ? 1 : (threads > 256 ? 256 : threads);
  return s->threads;
}
