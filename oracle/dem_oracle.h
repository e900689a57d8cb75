/*
 * dem_oracle.h -- CPU restatement of the MFiX DEM particle step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA library is checked
 * against: a C++ restatement, in the serial reference's operation order, of
 * the Fortran routines of model/des that form the DEM step.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.  The
 * product never links, loads or calls it.
 *
 * Parity is pinned against the reference's own golden tables
 * (tests/dem/DEM01..DEM06/AUTOTEST) by tests/test_oracle_golden.py.
 *
 * The API mirrors include/dem_b200.h with an orc_ prefix so the parity tests
 * can drive both sides with the same arrays (Fortran layouts, 1-based indices
 * at the boundary).
 */
#ifndef DEM_ORACLE_H
#define DEM_ORACLE_H

#include <stdint.h>
#include "../include/dem_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_handle orc_handle;

int  orc_create(const dem_params* p, int32_t max_pip, orc_handle** out);
int  orc_destroy(orc_handle* h);
const char* orc_last_error(const orc_handle* h);
/* Threads used by the OpenMP timing mode (1 = serial parity mode). */
int  orc_set_threads(orc_handle* h, int32_t nthreads);

int  orc_set_walls(orc_handle* h, const double* vertex, const double* norm_face, int32_t n_facets);
int  orc_upload_state(orc_handle* h, const double* pos, const double* vel, const double* omega,
                      const double* radius, const double* pmass, const double* omoi,
                      const int8_t* state, const int32_t* phase, int32_t max_pip);
int  orc_download_state(orc_handle* h, double* pos, double* vel, double* omega,
                        int8_t* state, int32_t max_pip);
int  orc_download_forces(orc_handle* h, double* fc, double* tow, int32_t max_pip);
int  orc_set_ab2_history(orc_handle* h, const double* acc_old, const double* rot_acc_old,
                         int32_t first_pass, int32_t max_pip);
int  orc_get_ab2_history(orc_handle* h, double* acc_old, double* rot_acc_old, int32_t max_pip);
int  orc_pair_count(orc_handle* h, int64_t* n_pairs);
int  orc_download_pairs(orc_handle* h, int32_t* neighbor_index, int32_t* neighbors,
                        double* pft, int64_t capacity, int32_t max_pip);
int  orc_upload_pairs(orc_handle* h, const int32_t* neighbor_index, const int32_t* neighbors,
                      const double* pft, int64_t n_pairs, int32_t max_pip);
int  orc_download_wall_history(orc_handle* h, int32_t* facet_id, double* pft, int32_t max_pip);
int  orc_upload_wall_history(orc_handle* h, const int32_t* facet_id, const double* pft, int32_t max_pip);
int  orc_set_outflow_bcs(orc_handle* h, const dem_outflow_bc* bcs, int32_t n);
int  orc_set_inflow_bcs(orc_handle* h, const dem_inflow_bc* bcs, int32_t n, uint64_t seed);
int  orc_push_inflow_random(orc_handle* h, const double* r, int64_t n);
int  orc_get_inflow_state(orc_handle* h, int32_t bc, int32_t* vacancy, double* mi_time);
int  orc_download_cells(orc_handle* h, int32_t* dg_pijk, int32_t max_pip);
/* facets_at_dg as CSR over 1-based DES cells: start[ncell2+1], ids (1-based) */
int  orc_download_facet_bins(orc_handle* h, int32_t* start, int32_t* ids, int32_t capacity,
                             int32_t* ncell2_out);
int  orc_download_edge_flags(orc_handle* h, int8_t* flags /* (nf,4): edge 0..3 */);

int  orc_desgrid_pic(orc_handle* h);
int  orc_neighbour(orc_handle* h);
int  orc_calc_force(orc_handle* h);
int  orc_cfnewvalues(orc_handle* h);
int  orc_init_neighbors(orc_handle* h);
int  orc_step(orc_handle* h, int32_t nn_first, int32_t nsteps);
int  orc_get_stats(orc_handle* h, dem_stats* out);

/* Coupling (GARG_2012 / Gidaspow / mean fields). */
int  orc_set_gas_fields(orc_handle* h, const dem_fluid_grid* g, const double* ep_g,
                        const double* u_g, const double* v_g, const double* w_g,
                        const double* p_force);
int  orc_get_mean_fields(orc_handle* h, double* ep_g, double* rop_s);
int  orc_comp_mean_fields(orc_handle* h);
int  orc_drag_gs_des0(orc_handle* h);
int  orc_drag_gs_gas0(orc_handle* h, double* f_gds, double* drag_am, double* drag_bm,
                      double* f_gp);
int  orc_drag_gs_des1(orc_handle* h);
int  orc_drag_gs_gas1(orc_handle* h, double* f_gds, double* drag_bm, double* f_gp);
int  orc_step_coupled(orc_handle* h, int32_t nn_first, int32_t nsteps);

/* Contact constants as CHECK_SOLIDS_DEM_COLL_LSD / _HERTZ derive them
 * (model/check_data/check_solids_dem.f:519-1122).  Inputs per phase:
 * d_p0, ro_s0 (reference size/mass: min over particles is applied by the
 * caller through ref_radius/ref_mass), e_young, v_poisson, en (M x M
 * row-major, DEM_MAX_PHASES stride), et, en_w, et_w, ew_young, vw_poisson,
 * kt_fac, kt_w_fac, des_etat_fac, des_etat_w_fac.  Fills the tables of *p and
 * p->dtsolid = tcoll / dtsolid_factor.  Returns tcoll through *tcoll_out. */
int  orc_contact_constants(dem_params* p, const double* ref_radius, const double* ref_mass,
                           const double* e_young, const double* v_poisson,
                           const double* en, const double* et,
                           const double* en_w, const double* et_w,
                           double ew_young, double vw_poisson,
                           double kt_fac, double kt_w_fac,
                           double des_etat_fac, double des_etat_w_fac,
                           double dtsolid_factor, double* tcoll_out);

#ifdef __cplusplus
}
#endif

#endif
