/*
 * dem_b200.h -- C ABI of the B200-native MFiX DEM particle step.
 *
 * This is the drop-in boundary for the DEM hot path of MFiX
 * (model/des).  In the reference the path is a sequence of argument-less
 * Fortran subroutines that share the module globals of `discretelement`
 * and are called in order by DES_TIME_STEP (model/des/des_time_march.f:293-460).
 * Each entry point below replaces one of those calls; a Fortran driver binds
 * them through ISO_C_BINDING (see the INTEGRATION notes) and passes its own
 * arrays, which keep their Fortran layout:
 *
 *   - per-particle vectors are (MAX_PIP,3) column-major: the x, y and z
 *     columns are three contiguous blocks of MAX_PIP doubles;
 *   - particle, pair and facet indices are 1-based at this boundary;
 *   - PFT_NEIGHBOR is (3,P): the three components of one pair are adjacent.
 *
 * Every function returns 0 on success or a DEM_ERR_* code; dem_last_error()
 * returns the message of the last failure on a handle.  Device state is
 * resident and authoritative between calls; the host arrays stay owned by
 * the caller and are only read or written inside upload/download calls.
 * Calls on one handle must come from one host thread at a time.
 */
#ifndef DEM_B200_H
#define DEM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DEM_ABI_VERSION 2

/* Maximum number of DEM solids phases (MFiX DIM_M is 10; DEM cases use few). */
#define DEM_MAX_PHASES 8

/* DES_COLL_MODEL_ENUM (model/des/discretelement_mod.f:196-200) */
#define DEM_COLL_LSD    0
#define DEM_COLL_HERTZ  1

/* DES_INTG_METHOD (model/des/discretelement_mod.f:205-207) */
#define DEM_INTG_EULER  0
#define DEM_INTG_AB2    1

/* Contact-force arithmetic. FP64 reproduces CALC_FORCE_DEM in double
 * precision with the serial reference's summation order.  SPLIT computes the
 * relative displacement, overlap and forces in FP32 from FP64 positions,
 * accumulates with compensated FP32 sums, and keeps FP64 integration and
 * FP64 tangential history. */
#define DEM_PREC_FP64   0
#define DEM_PREC_SPLIT  1

/* PARTICLE_STATE values (model/des/discretelement_mod.f:70-78) */
#define DEM_STATE_NONEXISTENT   0
#define DEM_STATE_NORMAL        1
#define DEM_STATE_ENTERING      2
#define DEM_STATE_EXITING       3
#define DEM_STATE_RIGID         10
#define DEM_STATE_NORMAL_GHOST  101

/* Error codes */
#define DEM_OK                   0
#define DEM_ERR_ARG              1   /* bad argument or size */
#define DEM_ERR_CUDA             2   /* a CUDA call failed */
#define DEM_ERR_ZERO_DISTANCE    3   /* two particle centres coincide (calc_force_dem.f:267-271) */
#define DEM_ERR_PAIR_OVERFLOW    4   /* pair list capacity exceeded; call again after growth */
#define DEM_ERR_WALL_SLOTS       5   /* more than COLLISION_ARRAY_MAX wall contacts on a particle */
#define DEM_ERR_ROGUE            6   /* NORMAL particle in a ghost cell with remove_rogue = 0 */
#define DEM_ERR_NONFINITE        7   /* NaN/Inf found in particle state */
#define DEM_ERR_STATE            8   /* call out of order (e.g. step before upload) */
#define DEM_ERR_TIMEOUT          9   /* a bounded host wait expired */
#define DEM_ERR_CAPACITY        10   /* a fixed-size buffer is too small */

/*
 * Parameters.  These mirror the DES namelist keywords and the derived
 * tables that CHECK_SOLIDS_DEM computes (model/check_data/check_solids_dem.f:
 * 519-782 for LSD, 798-1122 for Hertz) and the DES grid that DESGRID_INIT
 * builds (model/des/desgrid_mod.f:506-865) for a single rank.  Phase tables
 * are (M,L) row-major with stride DEM_MAX_PHASES, 0-based phases.
 */
typedef struct dem_params {
    int32_t n_phases;            /* DES_MMAX */
    int32_t coll_model;          /* DEM_COLL_* */
    int32_t intg_method;         /* DEM_INTG_* */
    int32_t neighbor_search_n;   /* NEIGHBOR_SEARCH_N */
    int32_t force_precision;     /* DEM_PREC_* */
    int32_t remove_rogue;        /* REMOVE_ROGUE_PARTICLES */
    int32_t no_k;                /* 2-D case (NO_K) */
    int32_t periodic[3];         /* DES_PERIODIC_WALLS_X/Y/Z */
    int32_t dg_imax, dg_jmax, dg_kmax;   /* interior DES grid cells per axis */
    int32_t collision_array_max; /* wall-history slots per particle (COLLISION_ARRAY_MAX, default 8) */
    int32_t reserved_i[6];

    double factor_rlm;           /* FACTOR_RLM (its default is the REAL(4) literal 1.2) */
    double dtsolid;              /* DTSOLID */
    double grav[3];              /* GRAV */
    double kn, kt, kn_w, kt_w;   /* LSD spring constants */
    double mew, mew_w;           /* sliding friction, particle-particle and particle-wall */
    double mew_r, mew_rw;        /* rolling friction */
    double max_radius;           /* MAX_RADIUS */
    double dg_xstart, dg_ystart, dg_zstart;  /* DES grid origin (dg_xstart...) */
    double dg_dxinv, dg_dyinv, dg_dzinv;     /* inverse DES cell widths */
    double domain_lo[3];         /* X_MIN, Y_MIN, Z_MIN */
    double domain_hi[3];         /* X_MAX, Y_MAX, Z_MAX */
    double des_etan[DEM_MAX_PHASES * DEM_MAX_PHASES];  /* particle-agnostic damping */
    double des_etat[DEM_MAX_PHASES * DEM_MAX_PHASES];
    double hert_kn[DEM_MAX_PHASES * DEM_MAX_PHASES];   /* Hertz spring factors / sqrt(R_eff) */
    double hert_kt[DEM_MAX_PHASES * DEM_MAX_PHASES];
    double des_etan_wall[DEM_MAX_PHASES];
    double des_etat_wall[DEM_MAX_PHASES];
    double hert_kwn[DEM_MAX_PHASES];
    double hert_kwt[DEM_MAX_PHASES];
    double reserved_d[8];
} dem_params;

/* Statistics (model/des/des_granular_temperature.f:33-267 and the contact
 * count of calc_force_dem.f:740-801). */
typedef struct dem_stats {
    int64_t n_normal;        /* NORMAL particles */
    int64_t n_pairs;         /* half-list pairs (entries of NEIGHBORS) */
    int64_t n_contacts;      /* pairs in contact at the last force evaluation */
    int64_t n_wall_contacts; /* particle-facet contacts at the last force evaluation */
    int64_t n_rogue_removed; /* particles deleted as rogue so far */
    int64_t steps_done;      /* DES_TIME_STEP calls executed on this handle */
    double  mean_vel[3];     /* mean particle velocity (NORMAL particles) */
    double  gran_temp[3];    /* <(v - <v>)^2> per component */
    double  kinetic_energy;  /* sum 0.5 m v^2 */
    double  max_overlap_ratio; /* max overlap / R_LM over contacts */
    double  bed_height;      /* mass-weighted mean y of NORMAL particles */
    double  s_time;          /* accumulated solids time S_TIME */
    int64_t n_outflow_removed; /* particles deleted by outflow boundaries so far */
    int64_t n_inflow_added;    /* particles seeded by mass-inflow boundaries so far */
    int64_t n_candidate_lists; /* candidate lists the pair build made so far (single
                                  systems without flow boundaries; no counterpart) */
    int64_t n_builds_filtered; /* pair builds that filtered a candidate list instead
                                  of scanning the DES grid (no counterpart) */
} dem_stats;

typedef struct dem_handle dem_handle;

/* ---- lifetime ---------------------------------------------------------- */

/* Allocates device state for max_pip particles (MAX_PIP) on the current CUDA
 * device.  Replaces the DES allocation in des_allocate_mod.f and the constant
 * set-up of CHECK_SOLIDS_DEM (the derived tables are taken from *p).
 * Limits: max_pip < 2^27; at most 1021 interior DES cells along x and z and
 * 4093 along y (DEM_ERR_ARG otherwise). */
int dem_create(const dem_params* p, int32_t max_pip, dem_handle** out);
int dem_destroy(dem_handle* h);
const char* dem_last_error(const dem_handle* h);
int dem_abi_version(void);

/* ---- geometry ---------------------------------------------------------- */

/* Wall facets: VERTEX(3,3,F) and NORM_FACE(3,F) of cartesian_grid/stl_mod.f:21-23
 * in Fortran layout (vertex[v + 3*c + 9*f]).  Bins them to the DES grid as
 * BIN_FACETS_TO_DG (model/des/stl_preproc_des_mod.f:135-203, TRI_BOX_OVERLAP
 * in stl_functions_des_mod.f:280-536) and flags edges shared by near-coplanar
 * facets as FLAG_FACETS_WHERE_EDGE_COLLISION_IS_IGNORED (stl_preproc_des_mod.f:
 * 361-490) does.  n_facets may be 0. */
/* DTSOLID of the following steps.  A coupled driver shortens the last DEM
 * step of each fluid step so the solids time lands on the fluid time
 * (DTSOLID = TIME + DT - S_TIME, des_time_march.f:308-314) and puts the
 * original value back after the fluid step (DES_TIME_END,
 * des_time_march.f:470-476).  Single-system handles; dt > 0. */
int dem_set_dtsolid(dem_handle* h, double dtsolid);

int dem_set_walls(dem_handle* h, const double* vertex, const double* norm_face,
                  int32_t n_facets);

/* ---- particle state ---------------------------------------------------- */

/* Copies the DES arrays in: DES_POS_NEW, DES_VEL_NEW, OMEGA_NEW (max_pip,3),
 * DES_RADIUS, PMASS, OMOI (max_pip), PARTICLE_STATE (int8) and the 1-based
 * solids phase PIJK(:,5). (model/des/discretelement_mod.f:387-391,579-588)
 * After a first full upload, radius, pmass, omoi, state and phase may each
 * be NULL: the handle keeps its own (a driver that changed only positions,
 * velocities and spins sends those).  Such a motion-only upload adds the
 * largest move of a particle to the bound the pair build and the gap
 * screens keep; any other upload clears them until the next build.  The
 * host arrays may be reused when the call returns. */
int dem_upload_state(dem_handle* h, const double* pos, const double* vel,
                     const double* omega, const double* radius,
                     const double* pmass, const double* omoi,
                     const int8_t* state, const int32_t* phase, int32_t max_pip);

/* Copies DES_POS_NEW, DES_VEL_NEW, OMEGA_NEW and PARTICLE_STATE out.
 * Any pointer may be NULL to skip that array. */
int dem_download_state(dem_handle* h, double* pos, double* vel, double* omega,
                       int8_t* state, int32_t max_pip);

/* FC and TOW (max_pip,3) as left by the last dem_calc_force call. */
int dem_download_forces(dem_handle* h, double* fc, double* tow, int32_t max_pip);

/* The Adams-Bashforth history DES_ACC_OLD / ROT_ACC_OLD (max_pip,3) and the
 * CFNEWVALUES first-pass flag, for restart hand-over. */
int dem_set_ab2_history(dem_handle* h, const double* acc_old,
                        const double* rot_acc_old, int32_t first_pass, int32_t max_pip);
int dem_get_ab2_history(dem_handle* h, double* acc_old, double* rot_acc_old,
                        int32_t max_pip);

/* ---- pair list ----------------------------------------------------------- */

/* Number of entries in NEIGHBORS after the last build. */
int dem_pair_count(dem_handle* h, int64_t* n_pairs);

/* NEIGHBOR_INDEX(max_pip) (1-based end pointers: row LL spans
 * NEIGHBOR_INDEX(LL-1) .. NEIGHBOR_INDEX(LL)-1, row 1 starts at 1),
 * NEIGHBORS(P) (1-based particle indices) and PFT_NEIGHBOR(3,P), in the order
 * of the serial reference build (desgrid_mod.f:1002-1299).  Any output pointer
 * may be NULL. capacity is the length of neighbors (pft holds 3*capacity). */
int dem_download_pairs(dem_handle* h, int32_t* neighbor_index, int32_t* neighbors,
                       double* pft, int64_t capacity, int32_t max_pip);

/* Installs a pair list with tangential history (restart / hand-over from the
 * CPU solver, write_res0_des.f:177-182).  The rows must be a valid half list. */
int dem_upload_pairs(dem_handle* h, const int32_t* neighbor_index,
                     const int32_t* neighbors, const double* pft,
                     int64_t n_pairs, int32_t max_pip);

/* Wall tangential history WALL_COLLISION_FACET_ID(cmax, max_pip) (1-based
 * facet ids, -1 free) and WALL_COLLISION_PFT(3, cmax, max_pip)
 * (model/des/discretelement_mod.f:637-642). */
int dem_download_wall_history(dem_handle* h, int32_t* facet_id, double* pft,
                              int32_t max_pip);

/* Restores the wall tangential history from the same arrays (a restart or a
 * hand-over from the CPU solver).  Facet ids must be -1 or 1..n_facets of
 * the facets installed by dem_set_walls.  Call after dem_upload_state, which
 * keeps the previous history. */
int dem_upload_wall_history(dem_handle* h, const int32_t* facet_id, const double* pft,
                            int32_t max_pip);

/* ---- restart files (model/des/write_res0_des.f, read_res0_des.f) -------- */

/* Scalars of a DEM restart file (RES, serial layout: 512-byte big-endian
 * records as WRITE_RES0_DES writes them). */
typedef struct dem_res_info {
    double  version;            /* read: the file's VERSION (written: 1.2 as a REAL(4) literal) */
    double  dtsolid;            /* DTSOLID stored in the file */
    int32_t vtp_findex;         /* VTP_FINDEX */
    int32_t tecplot_findex;     /* TECPLOT_FINDEX */
    int32_t n_particles;        /* read: existing non-ghost particles in the file */
    int32_t n_pairs;            /* read: pair entries in the file */
    double  ro_sol[DEM_MAX_PHASES];  /* write: RO_SOL of each phase's particles */
    double  reserved[4];
} dem_res_info;

/* WRITE_RES0_DES (write_res0_des.f:44-208) for a DEM run without MPPIC,
 * thermal, species, user variables, SuperDEM, glued spheres or mass
 * inflow: particle arrays of the existing non-ghost particles in slot order
 * (global id = 1-based slot), then the pair list.  The second pair array
 * holds each entry's owner (the reference writes a value its reader does not
 * use), so that dem_read_res0_des can restore the pair list exactly. */
int dem_write_res0_des(dem_handle* h, const char* path, const dem_res_info* info);

/* READ_RES0_DES (read_res0_des.f): particles into slots 1..n_particles
 * (the rest NONEXISTENT), PMASS/OMOI from DES_RADIUS and RO_SOL as
 * MAKE_ARRAYS_DES computes them (make_arrays_des.f:287-291), uploaded as
 * dem_upload_state does.  restore_pairs = 1 also uploads the pair list and
 * its tangential history (files from dem_write_res0_des); with 0 the pair
 * section is skipped and the caller builds the list (dem_init_neighbors), as
 * for files written by the reference.  Wall-contact and Adams-Bashforth
 * histories are not part of the format: restore them with
 * dem_upload_wall_history / dem_set_ab2_history when they were saved. */
int dem_read_res0_des(dem_handle* h, const char* path, int32_t restore_pairs, dem_res_info* info);

/* The record codec behind the two calls, on host arrays (no device needed).
 * dem_res_write takes the DES arrays in Fortran layout with 1-based
 * NEIGHBOR_INDEX/NEIGHBORS as dem_download_pairs returns them.
 * dem_res_read with pos == NULL reads the header only (counts into *info);
 * otherwise it fills max_pip slots and, when pair_owner is not NULL, the
 * pair entries as 1-based local owner/neighbour indices and PFT (3,P). */
int dem_res_write(const char* path, const dem_res_info* info, int32_t max_pip, int32_t no_k,
                  const double* pos, const double* vel, const double* omega, const double* radius,
                  const int8_t* state, const int32_t* phase, const int32_t* neighbor_index,
                  const int32_t* neighbors, const double* pft, int64_t n_pairs);
int dem_res_read(const char* path, dem_res_info* info, int32_t max_pip, int32_t no_k,
                 double* pos, double* vel, double* omega, double* radius, double* ro_sol,
                 int8_t* state, int32_t* phase, int32_t* pair_owner, int32_t* pair_neighbor,
                 double* pft, int64_t pair_cap);

/* ---- outflow boundaries (model/des/mass_outflow_dem.f) ------------------- */

/* One DEM outflow boundary (an entry of DEM_BCMO_MAP).  The DES cells it
 * watches are the box dg_lo..dg_hi (DES-grid indices as DG_FUNIJK takes
 * them: I_w..I_e, J_s..J_n, K_b..K_t of SET_BC_DEM_MO, set_bc_dem_mo.f:
 * 79-101, from IofBCPOS of the BC extents); a particle belongs to it when its
 * DES cell of the last DESGRID_PIC is in the box (DG_PIC).  `face` is the
 * plane the distance is measured from: YN(BC_J_s-1) for 'S', YN(BC_J_s) for
 * 'N', XE(BC_I_w-1) for 'W', XE(BC_I_w) for 'E', ZT(BC_K_b-1) for 'B',
 * ZT(BC_K_b) for 'T' (mass_outflow_dem.f:96-103). */
typedef struct dem_outflow_bc {
    int32_t plane;             /* BC_PLANE: 'N','S','E','W','T','B' */
    int32_t mass_outflow;      /* 1: BC_TYPE MASS_OUTFLOW (exiting particles take vel); 0: P_/OUTFLOW */
    int32_t dg_lo[3], dg_hi[3];
    int32_t reserved_i[4];
    double  face;
    double  vel[DEM_MAX_PHASES][3];   /* BC_U_s, BC_V_s, BC_W_s of each phase (MASS_OUTFLOW) */
    double  reserved_d[4];
} dem_outflow_bc;

/* Installs the outflow boundaries (n = 0 removes them).  Each DES_TIME_STEP
 * then runs UPDATE_EXIT_DES_VEL before CFNEWVALUES (des_time_march.f:
 * 372-375; FREEZE_EXIT_DES_VEL = .FALSE.) and MASS_OUTFLOW_DEM after it
 * (des_time_march.f:405): particles clear of the plane by more than their
 * radius become NORMAL, straddling ones EXITING (velocity frozen to the
 * normal component while moving out, or set to the boundary's for
 * MASS_OUTFLOW), and those past it are deleted, which forces the neighbour
 * search of that step.  Steps are then taken one at a time (no CUDA graph).
 * The boxes of the boundaries must not overlap. */
int dem_set_outflow_bcs(dem_handle* h, const dem_outflow_bc* bcs, int32_t n);

/* ---- mass inflow (model/des/mass_inflow_dem.f, layout_mi_dem.f) --------- */

/* One mass-inflow boundary: the seeding layout LAYOUT_MI_DEM builds
 * (DEM_MI(BCV_I), layout_mi_dem.f:96-420), the rate SET_BC_DEM_MI derives
 * (PI_COUNT, PI_FACTOR, set_bc_dem_mi.f:180-205) and the box of DES cells
 * SET_DEM_BCMI_IJK lists (set_bc_dem_mi.f:391-530).  The in-plane axes of
 * P and Q are x and z for 'N'/'S', y and z for 'E'/'W', x and y for 'T'/'B'
 * (SEED_NEW_PARTICLE, mass_inflow_dem.f:306-408). */
typedef struct dem_inflow_bc {
    int32_t plane;            /* BC_PLANE: 'N','S','E','W','T','B' */
    int32_t occupants;        /* DEM_MI%OCCUPANTS: seeding windows */
    int32_t vacancy;          /* DEM_MI%VACANCY: the next window, 1-based (1 after the layout) */
    int32_t pi_count;         /* PI_COUNT: particles per injection (0: none) */
    int32_t polydisperse;     /* DEM_MI%POLYDISPERSE */
    int32_t n_layout;         /* entries of poly_layout (NUMFRAC_LIMIT = 10000 in the reference) */
    int32_t dg_lo[3], dg_hi[3];   /* DES-cell box of the entering test (DEM_BCMI_IJK) */
    int32_t l_index;          /* DEM_MI%L: fluid-cell index along the normal (restart records only) */
    int32_t reserved_i[3];
    double  offset;           /* DEM_MI%OFFSET: the seeding coordinate along the normal */
    double  window;           /* DEM_MI%WINDOW */
    double  face;             /* plane of the entering test: YN(BC_J_s) for 'N', YN(BC_J_s-1) for 'S',
                                 XE(BC_I_w) for 'E', XE(BC_I_w-1) for 'W', ZT(BC_K_b) for 'T',
                                 ZT(BC_K_b-1) for 'B' (mass_inflow_dem.f:118-125) */
    double  pi_factor;        /* PI_FACTOR: solids steps per injection */
    double  mi_time;          /* DEM_MI_TIME: solids time of the next injection */
    double  start_time;       /* BC_MI_START_TIME */
    double  end_time;         /* BC_MI_END_TIME */
    const double*  p;         /* [occupants] DEM_MI%P: window corners on the first in-plane axis */
    const double*  q;         /* [occupants] DEM_MI%Q: on the second (ignored when NO_K) */
    const int32_t* poly_layout;   /* [n_layout] DEM_BC_POLY_LAYOUT: solids phase (1-based) per slot */
    const int32_t* w_cell;    /* [occupants] DEM_MI%W, or NULL (restart records only: written as 0) */
    const int32_t* h_cell;    /* [occupants] DEM_MI%H, or NULL (likewise) */
    double  d_p0[DEM_MAX_PHASES];   /* D_P0 of each phase */
    double  ro_s0[DEM_MAX_PHASES];  /* RO_S0 of each phase */
    double  vel[DEM_MAX_PHASES][3]; /* BC_U_s, BC_V_s, BC_W_s of each phase */
    double  reserved_d[4];
} dem_inflow_bc;

/* Installs the mass-inflow boundaries (n = 0 removes them; the arrays are
 * copied).  Each DES_TIME_STEP then runs MASS_INFLOW_DEM after CFNEWVALUES
 * and before MASS_OUTFLOW_DEM (des_time_march.f:404-405): ENTERING
 * particles of a boundary's cells that are clear of its plane by more than
 * their radius become NORMAL, and, once the solids time reaches DEM_MI_TIME
 * inside [BC_MI_START_TIME, BC_MI_END_TIME], PI_COUNT particles are seeded
 * in successive windows of the layout (random offsets inside the window,
 * the boundary's velocity, ENTERING) into the first NONEXISTENT slots, and
 * DEM_MI_TIME advances by PI_FACTOR*DTSOLID.  Each boundary draws three
 * uniform numbers per call, as RANDOM_NUMBER(RAND) does: first from the
 * queue that dem_push_inflow_random fills, then from the handle's own
 * generator (splitmix64 from `seed`).  DEM_ERR_CAPACITY when the handle has
 * no NONEXISTENT slot left.  Steps are then taken one at a time (no CUDA
 * graph); not available on a batch handle. */
int dem_set_inflow_bcs(dem_handle* h, const dem_inflow_bc* bcs, int32_t n, uint64_t seed);

/* Queues n uniform numbers in [0,1) for the inflow boundaries, in the order
 * MASS_INFLOW_DEM draws them (three per boundary per step): a Fortran host
 * passes the values of its own RANDOM_NUMBER stream to seed exactly as the
 * reference does. */
int dem_push_inflow_random(dem_handle* h, const double* r, int64_t n);

/* The current DEM_MI%VACANCY and DEM_MI_TIME of inflow boundary `bc`
 * (0-based), for restart files (read_res0_des.f:217). */
int dem_get_inflow_state(dem_handle* h, int32_t bc, int32_t* vacancy, double* mi_time);

/* One mass-inflow record of a RES file (write_res0_des.f:197-210,
 * read_res0_des.f:205-234): DEM_MI_TIME and DEM_MI's VACANCY, OCCUPANTS,
 * WINDOW, OFFSET and L; its W, H, P, Q arrays have `occupants` entries. */
typedef struct dem_res_inflow {
    double  mi_time;
    double  window;
    double  offset;
    int32_t vacancy;
    int32_t occupants;
    int32_t l_index;
    int32_t reserved;
} dem_res_inflow;

/* Reads the mass-inflow section at the end of a RES file: *n_bc receives
 * DEM_BCMI (0 for files without inflow); the records of the first max_bc
 * boundaries go to mi[], and, where w/hh/p/q are not NULL, their arrays to
 * row b of w/hh/p/q (max_occ entries per row; DEM_ERR_CAPACITY when a
 * boundary has more).  dem_write_res0_des writes the section of the
 * handle's inflow boundaries; dem_read_res0_des restores DEM_MI_TIME and
 * VACANCY into the boundaries installed on the handle when their number
 * matches the file's (RESTART_1 semantics). */
int dem_res_read_inflow(const char* path, int32_t no_k, int32_t* n_bc, dem_res_inflow* mi, int32_t max_bc,
                        int32_t* w, int32_t* hh, double* p, double* q, int32_t max_occ);

/* ---- particle output (model/des/vtp_mod.f) ------------------------------- */

/* One VTK region of particle data (the VTK_* keywords of a region). */
typedef struct dem_vtp_options {
    double  time;               /* TIMESTAMP, written in the header comment */
    int32_t angular_velocity;   /* VTK_PART_ANGULAR_VEL: also write Angular_velocity */
    int32_t use_box;            /* 0: the whole domain; 1: the box below */
    int32_t select_mode;        /* VTK_SELECT_MODE: 'C' centre inside, 'P' entirely inside, 'I' intersects */
    uint32_t phase_mask;        /* VTK_PART_PHASE: bit m-1 selects phase m; 0 = all phases */
    double  box_lo[3];          /* VTK_X_W, VTK_Y_S, VTK_Z_B */
    double  box_hi[3];          /* VTK_X_E, VTK_Y_N, VTK_Z_T */
    double  reserved[4];
} dem_vtp_options;

/* WRITE_VTP_FILE for particle data (vtp_mod.f:705-1257): a .vtp PolyData file
 * with coordinates, Diameter, Velocity (and Angular_velocity) of the NORMAL
 * particles the region selects, Float32 big-endian appended data as the
 * reference writes it.  opt may be NULL (whole domain, no spin).
 * *n_written (may be NULL) receives the number of particles written. */
int dem_write_vtp(dem_handle* h, const char* path, const dem_vtp_options* opt, int64_t* n_written);

/* The same writer on host arrays in Fortran layout (no device needed);
 * phase (1-based) may be NULL when phase_mask is 0. */
int dem_vtp_write(const char* path, const dem_vtp_options* opt, int32_t max_pip, const double* pos,
                  const double* vel, const double* omega, const double* radius, const int8_t* state,
                  const int32_t* phase, int64_t* n_written);

/* ---- per-stage entry points (one per reference call site) ----------------- */

/* DESGRID_PIC(.TRUE.) (desgrid_mod.f:877-995): cell of every particle and the
 * per-cell particle lists, and for periodic axes the wrap of particles that
 * crossed a periodic face (the self-exchange of DES_PAR_EXCHANGE). */
int dem_desgrid_pic(dem_handle* h);

/* DG_PIJK(max_pip), 1-based DES cell of each particle (0 for nonexistent). */
int dem_download_cells(dem_handle* h, int32_t* dg_pijk, int32_t max_pip);

/* NEIGHBOUR (neighbour.f:21-126): rebuild the pair list with
 * DESGRID_NEIGH_BUILD and carry the tangential history over. */
int dem_neighbour(dem_handle* h);

/* CALC_FORCE_DEM (calc_force_dem.f:18-544) including the wall contacts
 * CALC_DEM_FORCE_WITH_WALL_STL (calc_collision_wall_mod.f:54-794).
 * Stores FC and TOW on the device: the reference adds to FC/TOW, which
 * CFNEWVALUES leaves at zero, so within DES_TIME_STEP the two agree; a
 * second call without dem_cfnewvalues in between does not add up. */
int dem_calc_force(dem_handle* h);

/* CFUPDATEOLD + CFNEWVALUES (cfupdateold.f:15-46, cfnewvalues.f:641-864):
 * integrates with FC/TOW and zeroes them. */
int dem_cfnewvalues(dem_handle* h);

/* MAKE_ARRAYS_DES tail (make_arrays_des.f:348-406): DESGRID_PIC + NEIGHBOUR
 * on the uploaded positions. */
int dem_init_neighbors(dem_handle* h);

/* DES_TIME_STEP(NN) for NN = nn_first .. nn_first+nsteps-1 of a pure DEM
 * run (des_time_march.f:293-460): force, integrate, and the rebuild when
 * NN == 1 or mod(NN, NEIGHBOR_SEARCH_N) == 0.  Force and integration run as
 * one fused kernel; the result is identical to dem_calc_force followed by
 * dem_cfnewvalues. */
int dem_step(dem_handle* h, int32_t nn_first, int32_t nsteps);

/* dem_step replays whole NEIGHBOR_SEARCH_N-step periods as CUDA graphs when
 * the handle has a stream of its own (the default) and profiling is off.
 * on = 0 runs every step launch by launch. */
int dem_set_graphs(dem_handle* h, int32_t on);

/* Statistics of the current state. */
int dem_get_stats(dem_handle* h, dem_stats* out);

/* The statistics of dem_get_stats, bit for bit, computed without allocating
 * anything: no cudaMalloc or cudaFree and no host heap.  No counterpart in
 * the reference.  It is for callers that must not allocate while particles
 * are being stepped: cudaMalloc/cudaFree can synchronise the whole device and
 * so stall the streams of other handles on the same GPU, and a caller that
 * runs systems under a fixed device-memory budget cannot let a statistics
 * buffer grow with the system (dem_get_stats grows its buffer on demand).
 *
 * Its scratch is one static device array of the library, sized for
 * DEM_STATS_NOALLOC_MAX_PARTICLES particles (about 2 MiB, held on every GPU
 * that loads the library until the process exits).  Handles with more
 * particles get DEM_ERR_CAPACITY.  The first call made for a device looks up
 * the array's device address (cudaGetSymbolAddress); make that first call
 * before any stream capture begins.  All calls on a device share the array:
 * calls whose kernels overlap on the GPU (for example from two host threads
 * on handles with different streams) race and must be serialised by the
 * caller.  The call synchronises the handle's stream before it returns. */
#define DEM_STATS_NOALLOC_MAX_PARTICLES (1 << 23)
int dem_get_stats_noalloc(dem_handle* h, dem_stats* out);

/* Number of kernels this handle has launched so far (for launch accounting). */
int dem_launch_count(const dem_handle* h, int64_t* count);

/* Kernel-time accounting: when on, every kernel the handle launches is
 * bracketed by CUDA events on its stream and its time is added to one of
 * these classes. */
#define DEM_PROF_FORCE     0   /* contact force (+ fused integration) */
#define DEM_PROF_NEIGHBOR  1   /* pair-list build, history carry-over, transpose */
#define DEM_PROF_DESGRID   2   /* cell keys and per-cell lists */
#define DEM_PROF_INTEGRATE 3   /* stand-alone CFNEWVALUES */
#define DEM_PROF_COUPLING  4   /* drag and mean fields */
#define DEM_PROF_OTHER     5
#define DEM_PROF_WALLS     6   /* parts of DEM_PROF_FORCE: wall contacts, */
#define DEM_PROF_PAIRS     7   /* pair contacts, */
#define DEM_PROF_GATHER    8   /* per-particle sums (+ fused integration) */
#define DEM_PROF_N         9
/* on = 1: CUDA events around every kernel class; on = 2: also around the
 * parts of the force step (each part's events add launch gaps to it). */
int dem_set_profiling(dem_handle* h, int32_t on);
/* Milliseconds and launch counts per class since profiling was switched on
 * (synchronizes the handle's stream). */
int dem_get_profile(dem_handle* h, double* ms, int64_t* launches);

/* Sets the CUDA stream (cudaStream_t passed as void*) used by the handle.
 * NULL selects the legacy default stream.  The wall kernels of a force pass
 * run on a second stream of the handle's own, forked from and joined back
 * into this stream by events, so work ordered on this stream sees all of a
 * step's results. */
int dem_set_stream(dem_handle* h, void* stream);

/* Per-step force error of the split-precision path: max over particles of
 * |F_split - F_fp64| / max|F_fp64| for the current state (both computed,
 * nothing integrated). */
int dem_force_error(dem_handle* h, double* rel_err);

/* ---- CFD-DEM coupling (model/des/drag_gs_des0.f, comp_mean_fields0.f) ---- */

/* DES_INTERP_SCHEME (particle_filter.f): GARG_2012 selects COMP_MEAN_FIELDS0
 * and DRAG_GS_DES0/GAS0; NONE (the keyword's default) selects
 * COMP_MEAN_FIELDS1 and DRAG_GS_DES1/GAS1 without a filter (each particle
 * sees and feeds only its own fluid cell). */
#define DEM_INTERP_GARG 0
#define DEM_INTERP_NONE 1

/* DRAG_TYPE of DES_DRAG_GP (drag_gp_des.f:97-257).  GIDASPOW is the
 * reference's DRAG_GIDASPOW (drag_gs.f:536-598).  SINGLE_SPHERE is the
 * user drag law (DRAG_TYPE = 'USER_DRAG', drag_gp_des.f:169-171) that the
 * reference's terminal-velocity regression compiles in (tests/dem/DEM06,
 * usr_drag.f and usr_mod.f): DgA = 0.75*(RO_g*|u|/d_p)*Cd(Re) with the
 * Schiller-Naumann Cd = (24/Re)*(1 + 0.15*Re**0.687) (0 for Re = 0) and
 * Re = RO_g*usr_d_p0*|u|/MU_g from a fixed diameter usr_d_p0 (D_p0 of the
 * phase); independent of EP_g. */
#define DEM_DRAG_GIDASPOW      0
#define DEM_DRAG_SINGLE_SPHERE 1

/* Fluid grid description for the coupled step.  Uniform Cartesian grid of
 * imax x jmax x kmax interior cells starting at domain_lo with widths dx,dy,dz;
 * MFiX's IJK includes one ghost layer on every side. */
typedef struct dem_fluid_grid {
    int32_t imax, jmax, kmax;
    int32_t drag_model;          /* DEM_DRAG_GIDASPOW or DEM_DRAG_SINGLE_SPHERE */
    int32_t interp_scheme;       /* DES_INTERP_SCHEME: DEM_INTERP_GARG or DEM_INTERP_NONE */
    int32_t reserved_i;
    double dx, dy, dz;
    double ro_g, mu_g;           /* gas density and viscosity (uniform) */
    double ep_star;              /* packed-bed void fraction EP_STAR (for ep_s max) */
    double ur_f_gs;              /* under-relaxation of F_GP (drag_gp_des.f), usually 1 */
    double ro_s[DEM_MAX_PHASES]; /* RO_S0 of each solids phase (EP_S = ROP_S/RO_S) */
    double usr_d_p0;             /* Re diameter of DEM_DRAG_SINGLE_SPHERE */
    double reserved[5];
} dem_fluid_grid;

/* Installs the fluid grid and the gas fields on fluid cells (including
 * ghosts; (imax+2)*(jmax+2)*(kmax+2) values each in MFiX IJK order):
 * EP_G, U_G, V_G, W_G (staggered face velocities), and P_FORCE (3, ncells)
 * (may be NULL for zero). */
int dem_set_gas_fields(dem_handle* h, const dem_fluid_grid* g,
                       const double* ep_g, const double* u_g, const double* v_g,
                       const double* w_g, const double* p_force);

/* Reads the mean fields of the last deposition: EP_G and ROP_S per fluid cell. */
int dem_get_mean_fields(dem_handle* h, double* ep_g, double* rop_s);

/* PARTICLES_IN_CELL + COMP_MEAN_FIELDS (comp_mean_fields.f:30-40:
 * COMP_MEAN_FIELDS0 under DEM_INTERP_GARG, COMP_MEAN_FIELDS1 without a filter
 * under DEM_INTERP_NONE) + CALC_EPG_DES. */
int dem_comp_mean_fields(dem_handle* h);

/* CALC_DES_BEDHEIGHT (model/des/des_granular_temperature.f:201-267, the
 * formulation of Goldschmidt et al., Powder Technol. 138 (2003) 135-159):
 * per solids phase, sum(EP_S*h*VOL) / sum(EP_S*VOL) over the fluid cells
 * (ghost layers included) whose ROP_S of that phase is positive, h the
 * cell-centre height 0.5*(YN(J)+YN(J-1)) and EP_S = ROP_S/RO_S from the last
 * dem_comp_mean_fields (or coupled step).  Writes n_phases values; a phase
 * with no solids gives 0/0 as in the reference.  Needs dem_set_gas_fields
 * (a pure granular run installs its fluid grid with zero gas velocity). */
int dem_calc_des_bedheight(dem_handle* h, double* bed_height);

/* DRAG_GS_DES0 with GARG_2012 interpolation: adds the drag to FC.  Call after
 * dem_calc_force and before dem_cfnewvalues. */
int dem_drag_gs_des0(dem_handle* h);

/* DRAG_GS_GAS0 (model/des/drag_gs_des0.f:235-497), the gas-phase side of the
 * GARG_2012 drag that CALC_DES_2FLUID (calc_des_2fluid.f:70-73) calls from
 * the fluid solver: F_GP of every particle of a fluid cell again (with the
 * UR_F_GS under-relaxation of DES_DRAG_GP), its deposition to the nodes of
 * the particle's fluid cell, DRAG_AM = sum F_GP*W/DES_VOL_NODE and
 * DRAG_BM(:,c) = sum F_GP*V(c)*W/DES_VOL_NODE, and F_GDS per fluid cell as
 * the mean of its nodes' DRAG_AM (zero elsewhere).  Particles are binned by
 * the last PARTICLES_IN_CELL (dem_set_gas_fields, dem_comp_mean_fields,
 * dem_step_coupled).  Outputs, each optional (NULL = not copied): f_gds and
 * drag_am (ncells), drag_bm (ncells, 3) column-major as DRAG_BM, f_gp
 * (max_pip).  Serial, non-periodic fluid grid (DES_ADDNODEVALUES adds
 * nothing there). */
int dem_drag_gs_gas0(dem_handle* h, double* f_gds, double* drag_am, double* drag_bm, double* f_gp);

/* DRAG_GS_DES1 (model/des/drag_gs_des1.f:34-160) without a filter (the
 * DEM_INTERP_NONE case): per NORMAL particle the gas velocity at the centre
 * of its fluid cell (CALC_CELL_CENTER_GAS_VEL, drag_gs_des1.f:313-370), F_GP
 * by DES_DRAG_GP, FC += F_GP*(u_g - v_p) + P_FORCE*PVOL; F_GP = 0 for a
 * particle outside the fluid cells.  Call after dem_calc_force. */
int dem_drag_gs_des1(dem_handle* h);

/* DRAG_GS_GAS1 (model/des/drag_gs_des1.f:179-301) without a filter: F_GP of
 * every NORMAL particle of a fluid cell again, DRAG_BM(IJK,:) = sum
 * F_GP*V/VOL and F_GDS(IJK) = sum F_GP/VOL over the cell's particles (zero
 * elsewhere).  Outputs as dem_drag_gs_gas0 (each may be NULL); there is no
 * DRAG_AM in this scheme. */
int dem_drag_gs_gas1(dem_handle* h, double* f_gds, double* drag_bm, double* f_gp);

/* One coupled DES_TIME_STEP sequence: force, drag, integrate, rebuild if due,
 * particles-in-cell and mean fields. */
int dem_step_coupled(dem_handle* h, int32_t nn_first, int32_t nsteps);

/* ---- launch-shape autotuning (no counterpart in the reference) -------- */
typedef struct dem_tuning {
    int32_t pair_threads;        /* pair kernel: threads per block */
    int32_t pair_blocks_per_sm;  /* pair kernel: blocks per SM of its persistent grid */
    int32_t gather_threads;      /* gather kernel: threads per block */
    int32_t neigh_threads;       /* pair-build scan: threads per block */
    double  pair_ms, gather_ms, neigh_ms;  /* measured time of the chosen shapes (autotune only) */
    double  reserved[4];
} dem_tuning;

/* Times the candidate launch shapes of the hot kernels on the handle's
 * current state (reps launches each, CUDA events on its stream) and keeps
 * the fastest; results do not depend on the shapes.  Needs a state and a
 * pair list (after dem_init_neighbors / dem_sys_start). */
int dem_autotune(dem_handle* h, int32_t reps, dem_tuning* out);
int dem_get_tuning(dem_handle* h, dem_tuning* out);
int dem_set_tuning(dem_handle* h, const dem_tuning* in);

/* ---- batches of independent systems ----------------------------------
 * No counterpart in the reference, which runs one system per process.  A
 * batch handle holds many independent dry DEM systems of any sizes; every
 * kernel of a step runs once over all of them, each particle with its own
 * system's parameters (DES grid, walls, contact constants, DTSOLID, NN).
 * All systems of a batch share the collision model, the integrator, the
 * force precision and COLLISION_ARRAY_MAX (those of the parameters given to
 * dem_batch_create).  Each system rebuilds its pair list by its own NN rule
 * (NN == 1 or mod(NN, NEIGHBOR_SEARCH_N) == 0), so its results are the same
 * as in a handle of its own, whatever else runs in the batch.  Systems can
 * be added and removed between steps (their particle, cell, facet and bin
 * ranges are reserved from the limits below and never move while they
 * live).  The single-system calls (dem_upload_state, dem_step, ...) refuse a
 * batch handle; the coupling calls are not available on it. */
typedef struct dem_batch_limits {
    int32_t max_particles;     /* particles of all systems together */
    int32_t max_systems;       /* system slots (at most 65535) */
    int32_t max_cells;         /* DES-grid cells of all systems, plus 1 per system */
    int32_t max_search_cells;  /* search-grid cells of all systems */
    int32_t max_facets;        /* wall facets of all systems */
    int32_t max_facet_bins;    /* facet-in-cell entries of all systems */
    int32_t pairs_per_particle;/* pair-list room reserved per particle (0: 6); the
                                  list grows past it only when a build needs more */
    int32_t reserved[9];
} dem_batch_limits;

/* Device memory of a handle (dem_memory_info) or of a batch handle before
 * it is made (dem_batch_footprint).  No counterpart in the reference. */
typedef struct dem_memory {
    int64_t array_bytes;       /* the arrays sized by the particle, cell, facet and system
                                  counts (state, histories, grids, work arrays, tables) */
    int64_t pair_bytes;        /* the pair-list arrays at their capacity (with the
                                  pair build's candidate list on a single system) */
    int64_t scratch_bytes;     /* scan and staging scratch held now (grows on demand) */
    int64_t pair_capacity;     /* pairs the pair-list arrays hold */
    int64_t pairs;             /* pairs of the current list */
    int64_t reserved[3];
} dem_memory;

typedef struct dem_sys_status {
    int32_t capacity;          /* particles reserved for the system */
    int32_t started;           /* 1 once dem_sys_start has built its pair list */
    int32_t next_nn;           /* NN of its next DES_TIME_STEP */
    int32_t particle_offset;   /* first particle of its range in the handle */
    int64_t steps_done;
    double  s_time;
    double  reserved[6];
} dem_sys_status;

/* Cell ranges a system with parameters p takes from a batch: DES-grid cells
 * (with its end entry) and search-grid cells.  Host only, no device. */
int dem_params_cells(const dem_params* p, int32_t* des_cells, int32_t* search_cells);

/* The device memory dem_batch_create allocates for `common` and `lim`
 * (array_bytes + pair_bytes; scratch_bytes and pairs are 0).  Host only: it
 * counts the same arrays, in the same sizes, that creation allocates. */
int dem_batch_footprint(const dem_params* common, const dem_batch_limits* lim, dem_memory* out);
/* The device memory a handle holds now (any handle).  For a single-system
 * handle the wall, gas-field and boundary tables are not counted. */
int dem_memory_info(dem_handle* h, dem_memory* out);

/* Creates an empty batch handle on the current CUDA device.  `common` gives
 * the collision model, integrator, force precision and COLLISION_ARRAY_MAX
 * of all systems (its other fields are not used for the systems). */
int dem_batch_create(const dem_params* common, const dem_batch_limits* lim, dem_handle** out);

/* Adds a system with its own parameters and room for max_pip particles;
 * returns its id.  DEM_ERR_CAPACITY when the limits are exhausted. */
int dem_sys_add(dem_handle* h, const dem_params* p, int32_t max_pip, int32_t* sys);
/* Removes a system; its ranges become free for later systems. */
int dem_sys_remove(dem_handle* h, int32_t sys);
/* dem_set_walls / dem_upload_state / dem_download_state of one system
 * (arrays with max_pip rows, max_pip <= its capacity). */
int dem_sys_set_walls(dem_handle* h, int32_t sys, const double* vertex, const double* norm_face, int32_t nf);
int dem_sys_upload_state(dem_handle* h, int32_t sys, const double* pos, const double* vel,
                         const double* omega, const double* radius, const double* pmass,
                         const double* omoi, const int8_t* state, const int32_t* phase,
                         int32_t max_pip);
int dem_sys_download_state(dem_handle* h, int32_t sys, double* pos, double* vel, double* omega,
                           int8_t* state, int32_t max_pip);
/* Builds the first pair list of the given systems (dem_init_neighbors for
 * each) in one pass; the running systems keep theirs.  They then step from
 * NN = 1.  Every system with particles must be started before a step. */
int dem_sys_start(dem_handle* h, const int32_t* sys, int32_t n_sys);
/* nsteps DES_TIME_STEPs of every started system, each with its own NN. */
int dem_batch_step(dem_handle* h, int32_t nsteps);
/* Statistics of one system (contact counts are not kept per system: 0). */
int dem_sys_get_stats(dem_handle* h, int32_t sys, dem_stats* out);
/* dem_download_pairs of one system: its rows as its own 1-based CSR. */
int dem_sys_download_pairs(dem_handle* h, int32_t sys, int32_t* neighbor_index, int32_t* neighbors,
                           double* pft, int64_t cap, int32_t max_pip);
int dem_sys_info(dem_handle* h, int32_t sys, dem_sys_status* out);

#ifdef __cplusplus
}
#endif

#endif /* DEM_B200_H */
