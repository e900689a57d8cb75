// dem_internal.cuh -- shared definitions of the CUDA DEM library.
//
// Device layout (n = MAX_PIP):
//   pos4[b][i] = (x, y, z, radius)      double4, double-buffered (b = 0/1)
//   vel4[b][i] = (u, v, w, pmass)       double4, double-buffered
//   omg4[b][i] = (wx, wy, wz, omoi)     double4, one array (omg4[0] and
//                                       omg4[1] are the same): the spin is
//                                       updated in place, and a particle with
//                                       no torque under Euler is not touched
//   state[i]   int8 PARTICLE_STATE, phase[i] uint8 (0-based)
//   fc, tow    (n,3) column blocks, as FC/TOW of discretelement_mod.f:630
//   pairs      CSR half list: row_end[i] = pairs in rows 0..i,
//              nbrs[P] 0-based, pft[b][3P] (3,P) like PFT_NEIGHBOR,
//              and the transpose in_start[n+1] / in_pair[] = (owner, cc)
//              sorted by owner so each particle can gather the forces of
//              the pairs it does not own in the serial reference's order.
// Packing a particle's position with its radius (and velocity with mass,
// spin with inverse inertia) makes each neighbour gather one 32-byte sector
// per quantity.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <deque>
#include <string>
#include <vector>

#include "../../include/dem_b200.h"

namespace demb {

// Neighbours per particle kept by the count pass of the pair build.
constexpr int NSLOT = 16;
constexpr double SMALL_NUMBER = 1.0e-15;       // param1_mod.f:26
constexpr double UNDEFINED_D  = 9.87654321e31; // param1_mod.f:20
constexpr int MAXP = DEM_MAX_PHASES;

// Error word bits (device -> host)
enum : unsigned {
  EF_ZERO_DIST   = 1u << 0,
  EF_WALL_SLOTS  = 1u << 1,
  EF_PAIR_CAP    = 1u << 2,
  EF_ROGUE_FATAL = 1u << 3,
  EF_CELL_CAP    = 1u << 4,
  EF_NONFINITE   = 1u << 5,
  EF_INFLOW_CAP  = 1u << 6,   // fewer NONEXISTENT slots than particles to seed
};

// Per-pair flag bits (pflag) between force passes.
enum : uint8_t {
  PF_CONTACT = 1,   // in contact at the last force pass (its record is valid)
  PF_HIST    = 2,   // its tangential history PFT is nonzero
};

// The candidate list of a single-system handle's pair build (neighbor.cu):
// pairs within the search radius plus a skin, kept while the displacement
// bound since its build stays within half the skin.
struct CandState {
  double disp;  // displacement bound since the list was built
  int have;     // the list is complete (built, within its capacity)
  int ok;       // this build filters the list (set at the start of each build)
  int build;    // this build makes a new list
  int total;    // entries of the last list build
  int uses;     // builds that filtered the current list
  int cool;     // builds left before the next list is made (after one expired unused)
};

// Contacts of a split-precision pair pass whose onset-of-slip test lies
// near its threshold (force_split.cu): 2 * pair index + 1 when the pair
// had a history.  The count starts at zero and k_slip_fix, which follows
// every pass, clears it; past SLIP_FIX_CAP a contact keeps its FP32
// decision.
constexpr int SLIP_FIX_CAP = 4096;
struct SlipFix {
  unsigned count;
  unsigned pad;
  long long pair[SLIP_FIX_CAP];
};

struct DevErr {
  unsigned flags;
  int first_rogue;   // smallest rogue particle index of the last build (n if none)
  int zero_a, zero_b;  // particles of a zero-distance pair
  unsigned long long n_contacts;
  unsigned long long n_wall_contacts;
  unsigned long long rogue_removed;
  unsigned long long outflow_removed;
  int cand_lists;     // candidate lists built (complete) so far
  int cand_filtered;  // pair builds that filtered a candidate list so far
};

// Parameters as kernels see them (passed by value).
struct DevParams {
  int n;
  int coll, intg, nph, no_k, cmax, remove_rogue, first_pass, prec;
  int per[3];
  int istart1, iend1, istart2, iend2;
  int jstart1, jend1, jstart2, jend2;
  int kstart1, kend1, kstart2, kend2;
  int c1, c2, c3, ncell2;
  double dt, grav[3];
  double kn, kt, kn_w, kt_w, mew, mew_w, mew_r, mew_rw;
  double factor_rlm, max_radius;
  double dg_start[3], dg_inv[3];
  double lo[3], hi[3], L[3], inv_L[3];  // inv_L = 1 / L
  double etan[MAXP * MAXP], etat[MAXP * MAXP], hkn[MAXP * MAXP], hkt[MAXP * MAXP];
  double etanw[MAXP], etatw[MAXP], hkwn[MAXP], hkwt[MAXP];
  // FP32 copies for the split-precision pair force: HERT_KN, HERT_KT,
  // DES_ETAN*sqrt(HERT_KN), DES_ETAT*sqrt(HERT_KT) (Hertz), DES_ETAN,
  // DES_ETAT, KN, KT (linear spring-dashpot), MEW
  float hkn32[MAXP * MAXP], hkt32[MAXP * MAXP], etan_sq32[MAXP * MAXP], etat_sq32[MAXP * MAXP];
  float etan32[MAXP * MAXP], etat32[MAXP * MAXP];
  float kn32, kt32, mew32;
  // search grid of the pair build: fn[a] interior cells of width 1/f_inv[a]
  // over the DES-grid interior, plus one ghost layer on each side
  int fn[3], fc1, fc2, nfcell;
  double f_inv[3];
  // place of the system in a batch handle (0 for an ordinary handle):
  // particles [p_begin, p_end), DES cells from cell_off, search cells from
  // fcell_off in the handle-wide cell arrays; n stays the handle-wide count
  int p_begin, p_end, cell_off, fcell_off;
};

// Batch view of a kernel: the parameter block of every system and the
// system of every particle.  Kernels instantiated with B = false use the
// by-value block of the handle's single system and never touch the view.
struct BatchView {
  const DevParams* tab;       // [system]
  const uint16_t* sys_of;     // [particle]
  const uint8_t* due;         // [system] 1 = rebuild its pair list now, 2 = first build (no history)
  int* first_rogue;           // [system] smallest rogue particle of the last build
};

template <bool B>
__device__ __forceinline__ const DevParams& sysp(const DevParams& p, const BatchView& bv, int particle) {
  if constexpr (B) return bv.tab[bv.sys_of[particle]];
  else return p;
}

// What the two particles of a contact pair need to add the pair's terms to
// FC/TOW in the reference's order: FC_TMP, CROSS(NORMAL, FT) with the two
// lever arms (the torques are DIST_CL*TOW_force and DIST_CI*TOW_force), and
// KN_DES and OVERLAP_N for the rolling-friction torque.  80 bytes.
struct PairRec {
  double fc[3], tf[3], dcl2, dci2, kn, ov;
};

struct FacetBinEntry {  // one entry of facets_at_dg(cell)
  double mn, mx;        // facet extent along dir
  int id;               // 0-based facet
  int dir;              // 0-based axis of smallest extent
};

// ---------------------------------------------------------------------------
// Host-side handle
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

// Host bookkeeping of one system of a batch handle.
struct SysSlot {
  bool live = false;          // the slot holds a system
  bool clean = true;          // no rows of an earlier occupant left under this id
  bool started = false;       // its pair list exists and it steps
  bool have_state = false;
  dem_params prm;
  DevParams dp;               // p_begin/p_end/cell_off/fcell_off filled in
  int cap = 0;                // particles reserved (p_end - p_begin)
  int nn = 1;                 // NN of its next DES_TIME_STEP
  bool first_pass = true;
  long long steps_done = 0;
  double s_time = 0.0;
  int fac_off = 0, nf = 0;     // its wall facets in the handle-wide facet arrays
  int bin_off = 0, nbin = 0;   // its facet-bin entries
};

// First-fit allocator over an index range (particles or cells of a batch).
struct RangeAlloc {
  std::vector<std::pair<int, int>> free_;  // (begin, length), sorted by begin
  void reset(int total) { free_.assign(1, {0, total}); }
  int take(int len, int align);             // begin, or -1 when nothing fits
  void give(int begin, int len);
};

}  // namespace demb

struct dem_handle {
  dem_params prm;
  demb::DevParams dp;
  int n = 0;

  // batch of independent systems (dem_batch_create); empty otherwise
  std::vector<demb::SysSlot> sys;
  demb::RangeAlloc part_alloc, cell_alloc, fcell_alloc, fac_alloc, bin_alloc;
  int max_facets = 0, max_bins = 0;
  demb::DevParams* d_sys = nullptr;   // device copy of sys[*].dp
  uint16_t* sys_of = nullptr;         // [particle] system
  uint8_t* d_due = nullptr;           // 3 masks of max_systems: eager events, and the idle
                                      // and rebuild steps of a captured period
  const uint8_t* due_cur = nullptr;   // the mask the next kernels read
  int* d_first_rogue = nullptr;       // [system]
  int ncell_total = 0, nfcell_total = 0;
  int n_act = 0, nfc_act = 0;         // extent of the live systems' particle and search-cell ranges
  int n_built = 0;                    // the particle extent of the current pair list's build
  bool batch() const { return !sys.empty(); }
  // The particles and search cells the step kernels cover: for a batch the
  // extent of its live systems (the ranges past it belong to no system: no
  // particle exists there and no cell is read), else all of them.
  int nl() const { return batch() ? n_act : n; }
  int nfl() const { return batch() ? nfc_act : dp.nfcell; }
  demb::BatchView bview() const { return demb::BatchView{d_sys, sys_of, due_cur, d_first_rogue}; }
  int dev = 0;
  cudaStream_t stream = 0;
  std::string err;
  long long launches = 0;
  bool have_state = false, have_pairs = false;
  int cur = 0;  // current state buffer
  int pcur = 0; // current pft buffer
  bool first_pass = true;
  long long steps_done = 0;
  double s_time = 0.0;

  // particle state
  double4* pos4[2] = {nullptr, nullptr};
  double4* vel4[2] = {nullptr, nullptr};
  double4* omg4[2] = {nullptr, nullptr};
  int8_t* state = nullptr;
  uint8_t* phase = nullptr;
  double* fc = nullptr;   // (n,3)
  double* tow = nullptr;
  double* acc_old = nullptr;
  double* rot_acc_old = nullptr;

  // DES grid
  int* dg_pijk = nullptr;     // 1-based cell, 0 = none
  int* cell_cnt = nullptr;    // ncell2
  int* cell_start = nullptr;  // ncell2+1
  int* cell_fill = nullptr;   // ncell2
  int* cell_list = nullptr;   // n
  int* fcell_key = nullptr;   // n: search-grid cell of each particle (0-based)
  int* fcell_cnt = nullptr;   // nfcell+1
  int* fcell_start = nullptr; // nfcell+1
  int* fcell_list = nullptr;  // n
  double4* spos = nullptr;    // n: positions in search-cell order (pair build)
  float4* sposf = nullptr;    // n: the same rounded to FP32 (conservative distance pre-check)
  int4* sinfo = nullptr;      // n: (particle, packed DES cell (i,j,k), state, search cell) in that order
  uint32_t* nslot = nullptr;  // n * NSLOT: rows kept by the count pass of the pair build, by particle
  int* long_rows = nullptr;   // n + 1: sorted-copy places of the rows longer than NSLOT, count at [n]
  // candidate list (single-system handles): cand_end[i] ends particle i's
  // candidates in cand_nb (particle indices); cand_cnt / cand_start /
  // cand_fill are build scratch, qof[i] the particle's place in the sorted
  // copy (-1 when not in it)
  int* cand_end = nullptr;
  int* cand_cnt = nullptr;
  int* cand_start = nullptr;
  int* cand_fill = nullptr;
  int* qof = nullptr;
  int* cand_nb = nullptr;
  long long cand_cap = 0;
  demb::CandState* cand = nullptr;
  demb::SlipFix* slipfix = nullptr;  // split pair pass: contacts near the onset of slip

  // pairs
  long long pair_cap = 0;
  long long arr_bytes = 0;    // device bytes of the arrays sized by the counts (handle_arrays and the batch tables)
  long long n_pairs = 0;      // host copy of the pair count (valid when !np_stale)
  bool np_stale = false;      // the last build ran without reading the count back
  int* d_np = nullptr;        // device pair count (persistent pair kernels read it)
  int n_sm = 148;             // multiprocessors of the device
  // launch shapes of the hot kernels (dem_autotune picks them)
  struct Tune {
    int pair_threads = 256, pair_bpsm = 8;  // pair kernel: threads per block, resident blocks per SM
    int gather_threads = 256;               // gather kernel: threads per block
    int neigh_threads = 128;                // pair-build scan: threads per block
  } tune;
  bool capturing = false;     // inside a CUDA graph capture: no host syncs
  cudaStream_t own_stream = nullptr;
  // the wall kernels of a force pass run on side_stream beside the pair
  // kernel (they write disjoint arrays); ev_fork / ev_join order them
  cudaStream_t side_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaGraphExec_t graphs[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  long long graph_launches = 0;
  long long graph_kernels[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // kernels per graph replay
  bool no_graphs = false;
  int* row_cnt = nullptr;     // n
  int* row_end[2] = {nullptr, nullptr};   // n (current / previous build)
  int* nbrs[2] = {nullptr, nullptr};      // cap
  double* pft[2] = {nullptr, nullptr};    // 3*cap; pft[pcur] is current, the other takes the carry-over of a rebuild
  int* in_cnt = nullptr;      // n
  int* in_start = nullptr;    // n+1
  int* in_fill = nullptr;     // n
  int2* in_pair = nullptr;    // cap
  int* in_pos = nullptr;      // cap: slot of each pair in its neighbour's incoming list (inverse of in_pair)
  uint8_t* in_flag = nullptr; // cap: PF_CONTACT of the pair at each incoming slot (split-precision records)
  int* pair_owner = nullptr;  // cap
  // cap: PF_* bits of each pair, one array per history buffer: pflagb[pcur]
  // goes with pft[pcur] (the other is stencil-rank scratch during a build
  // and the output of a split-precision force pass)
  uint8_t* pflagb[2] = {nullptr, nullptr};
  uint8_t* pflag() const { return pflagb[pcur]; }
  uint8_t* touched = nullptr; // n: 1 = in some pair contact at the current force pass
  uint8_t* wall_hit = nullptr; // n: 1 = in some wall contact (its terms are in wf)
  float* pgap = nullptr;      // cap: gap |d| - (r_i + r_j) of each pair at the last build, rounded down
  double* skin = nullptr;     // [0]: bound on any particle's displacement since the last build
  unsigned* vslot = nullptr;  // [32]: per-step displacement bounds, as float bits
  demb::PairRec* prec = nullptr; // cap: contact terms of the last force pass
  int rb = 0;                 // which row_end/nbrs buffer is current

  // walls
  int nf = 0;
  double* vertex = nullptr;   // [f][v][c]
  double* norm_face = nullptr;// [f][c]
  int8_t* ignore_edge = nullptr; // [f][4]
  int* fbin_start = nullptr;  // ncell2+1
  demb::FacetBinEntry* fbin = nullptr;
  int n_fbin = 0;
  int* wall_fid = nullptr;    // [i][cmax]
  double* wall_pft = nullptr; // [i][cmax][3]
  uint8_t* wall_live = nullptr; // [i] 1 when some wall slot may be in use
  uint8_t* wall_cand = nullptr; // [i] 1 when the particle's DES cell holds facets
  int* wall_list = nullptr;     // this step's particles with wall work (arbitrary order)
  float* wgap = nullptr;        // [i] clearance from the facets of its DES cell at the last build
  // outflow boundaries (single handles): host copy, device copy, the
  // FIRST_PASS of UPDATE_EXIT_DES_VEL
  std::vector<dem_outflow_bc> obc;
  dem_outflow_bc* d_obc = nullptr;
  bool exit_first_pass = true;
  // mass-inflow boundaries (single handles): host copies with their layout
  // arrays, the device copy (membership and entering test), the queue and
  // generator of the uniform numbers, the particles seeded since the last
  // DESGRID_PIC (not yet in its cell lists) and the seed records
  struct Inflow {
    dem_inflow_bc bc;
    std::vector<double> p, q;
    std::vector<int32_t> layout;
    std::vector<int32_t> w, hh;  // DEM_MI%W, %H for restart records (zeros when not given)
  };
  std::vector<Inflow> ibc;
  dem_inflow_bc* d_ibc = nullptr;
  std::deque<double> irand;
  uint64_t irng = 0;
  uint8_t* pic_fresh = nullptr;
  void* d_seed = nullptr;
  int seed_cap = 0;
  long long inflow_added = 0;
  int* d_nwall = nullptr;       // their count
  double* wf = nullptr;       // [i][6] wall force and torque of the last force pass (valid with wall_hit)

  // scan scratch
  int* scan_tmp = nullptr;
  size_t scan_tmp_elems = 0;

  // error word
  demb::DevErr* derr = nullptr;
  demb::DevErr* herr = nullptr;   // pinned mirror

  // reductions for stats
  double* red = nullptr;      // scratch doubles
  int red_elems = 0;

  // coupling (see coupling.cu)
  struct Gas* gas = nullptr;

  // host<->device staging (kept between calls)
  void* stage = nullptr;
  size_t stage_bytes = 0;

  // kernel-time accounting (dem_set_profiling)
  int prof = 0;                // 0 off, 1 kernel classes, 2 also the parts of the force step
  struct ProfEv { int cls; cudaEvent_t a, b; };
  std::vector<ProfEv> prof_pending;
  std::vector<cudaEvent_t> ev_pool;
  double prof_ms[DEM_PROF_N] = {0};
  long long prof_n[DEM_PROF_N] = {0};
};

namespace demb {

// set by every API entry point on failure
int set_err(dem_handle* h, int code, const std::string& msg);
int check_cuda(dem_handle* h, cudaError_t e, const char* what);

// scan.cu: exclusive scan of n ints into out (out may alias in); total
// written to *d_total (device pointer) when non-null.
int exclusive_scan(dem_handle* h, const int* in, int* out, int n, int* d_total);

// desgrid.cu / neighbor.cu / force.cu / walls.cu host drivers
int run_desgrid_pic(dem_handle* h, bool sort_cells);
int run_neighbour(dem_handle* h, bool carry_history);
int run_force(dem_handle* h, bool fused);
int run_cfnewvalues(dem_handle* h);
int run_bin_facets(dem_handle* h, const double* vertex_fortran, const double* norm_fortran, int nf);
int run_split_force_error(dem_handle* h, double* rel_err);
void launch_pairs_split(dem_handle* h);         // force_split.cu
void launch_gather_split(dem_handle* h, int mode);
int ensure_pair_capacity(dem_handle* h, long long need);
int build_transpose(dem_handle* h, int nb);    // neighbor.cu
void launch_neigh_count(dem_handle* h, const int* skip = nullptr);        // neighbor.cu: count pass of the pair build
void set_hist_flags(dem_handle* h);            // neighbor.cu: PF_HIST from the current history
void launch_skin(dem_handle* h);               // force.cu: adds the step's displacement to the bound
void skin_unknown(dem_handle* h);              // force.cu: positions changed from outside: no pair skipped
void launch_wall_gaps(dem_handle* h);          // force.cu: wall clearances at a build (with the pair gaps)
int run_cfnewvalues_outflow(dem_handle* h, bool* force_nsearch);  // outflow.cu: exit velocities, CFNEWVALUES, MASS_OUTFLOW_DEM
int run_mass_inflow(dem_handle* h);  // inflow.cu: MASS_INFLOW_DEM (entering test, seeding)
void launch_wall_cand(dem_handle* h);          // desgrid.cu: facet-cell flag of every particle
void launch_pairs_only(dem_handle* h);         // force.cu: pair kernel of the handle's precision
void launch_gather_only(dem_handle* h);        // force.cu: gather kernel, forces into FC/TOW
// capi.cu: parameter block of a system with handle-wide particle count n
void fill_devparams(const dem_params& q, int n, DevParams& p);
bool des_grid_ok(const dem_params& q);
int alloc_handle(dem_handle* h, int nc, int nfc, long long pairs);
// Device bytes of the pair-list arrays for cap pairs (ensure_pair_capacity).
long long pair_array_bytes(long long cap);

// The arrays of a handle for n particles, nc DES cells and nfc search cells
// (COLLISION_ARRAY_MAX from h->dp), each given to A(&pointer, bytes): the
// allocation list of alloc_handle, and what dem_batch_footprint counts.
template <class F>
void handle_arrays(dem_handle* h, size_t n, size_t nc, size_t nfc, F&& A) {
  const size_t cmax = (size_t)h->dp.cmax;
  for (int b = 0; b < 2; ++b) {
    A((void**)&h->pos4[b], sizeof(double4) * n);
    A((void**)&h->vel4[b], sizeof(double4) * n);
    A((void**)&h->row_end[b], sizeof(int) * n);
  }
  // the spin is one array under both buffer names: only the integrating
  // gather of a particle writes it, after every kernel that reads it
  A((void**)&h->omg4[0], sizeof(double4) * n);
  h->omg4[1] = h->omg4[0];
  A((void**)&h->state, n);
  A((void**)&h->phase, n);
  A((void**)&h->fc, sizeof(double) * 3 * n);
  A((void**)&h->tow, sizeof(double) * 3 * n);
  A((void**)&h->acc_old, sizeof(double) * 3 * n);
  A((void**)&h->rot_acc_old, sizeof(double) * 3 * n);
  A((void**)&h->dg_pijk, sizeof(int) * n);
  A((void**)&h->cell_cnt, sizeof(int) * (nc + 1));
  A((void**)&h->cell_start, sizeof(int) * (nc + 1));
  A((void**)&h->cell_fill, sizeof(int) * (nc + 1));
  A((void**)&h->cell_list, sizeof(int) * n);
  A((void**)&h->fcell_key, sizeof(int) * n);
  A((void**)&h->fcell_cnt, sizeof(int) * (nfc + 1));
  A((void**)&h->fcell_start, sizeof(int) * (nfc + 1));
  A((void**)&h->fcell_list, sizeof(int) * n);
  A((void**)&h->spos, sizeof(double4) * n);
  A((void**)&h->sposf, sizeof(float4) * n);
  A((void**)&h->sinfo, sizeof(int4) * n);
  A((void**)&h->nslot, sizeof(uint32_t) * NSLOT * n);
  A((void**)&h->long_rows, sizeof(int) * (n + 1));
  A((void**)&h->row_cnt, sizeof(int) * n);
  A((void**)&h->in_cnt, sizeof(int) * n);
  A((void**)&h->in_start, sizeof(int) * (n + 1));
  A((void**)&h->in_fill, sizeof(int) * n);
  A((void**)&h->fbin_start, sizeof(int) * (nc + 1));
  A((void**)&h->wall_fid, sizeof(int) * cmax * n);
  A((void**)&h->wall_pft, sizeof(double) * 3 * cmax * n);
  A((void**)&h->wall_live, n);
  A((void**)&h->wf, sizeof(double) * 6 * n);
  A((void**)&h->touched, n);
  A((void**)&h->wall_hit, n);
  A((void**)&h->wall_cand, n);
  A((void**)&h->wall_list, sizeof(int) * n);
  A((void**)&h->wgap, sizeof(float) * n);
  A((void**)&h->d_nwall, sizeof(int));
  A((void**)&h->skin, sizeof(double));
  A((void**)&h->vslot, sizeof(unsigned) * 32);
  A((void**)&h->derr, sizeof(DevErr));
  A((void**)&h->d_np, sizeof(int));
  A((void**)&h->slipfix, sizeof(SlipFix));
  if (!h->batch()) {
    A((void**)&h->cand_end, sizeof(int) * n);
    A((void**)&h->cand_cnt, sizeof(int) * n);
    A((void**)&h->cand_start, sizeof(int) * (n + 1));
    A((void**)&h->cand_fill, sizeof(int) * n);
    A((void**)&h->qof, sizeof(int) * n);
    A((void**)&h->cand, sizeof(CandState));
  }
}
int upload_range(dem_handle* h, int off, int cnt, int nph, const double* pos, const double* vel,
                 const double* omega, const double* radius, const double* pmass, const double* omoi,
                 const int8_t* state, const int32_t* phase, bool note_moves = false);
int download_range(dem_handle* h, int off, int cnt, double* pos, double* vel, double* omega, int8_t* state);
int stats_range(dem_handle* h, int off, int cnt, dem_stats* s);
// walls.cu: facets of batch system `sys` binned to its DES cells
int run_bin_facets_sys(dem_handle* h, int sys, const double* vertex_fortran, const double* norm_fortran, int nf);
int fetch_errors(dem_handle* h);
void* stage_buffer(dem_handle* h, size_t bytes);
void free_gas(dem_handle* h);                   // coupling.cu
long long host_pairs(dem_handle* h);            // pair count on the host (syncs when stale)
void invalidate_graphs(dem_handle* h);

// Grid of the persistent kernels over the pair list: a fixed number of
// resident blocks.
inline unsigned pair_grid(const dem_handle* h, int threads) {
  return (unsigned)(h->n_sm * (2048 / threads));
}

// Brackets the kernels issued in its scope with CUDA events when the
// handle's profiling is on.
struct ProfScope {
  dem_handle* h;
  int idx = -1;
  ProfScope(dem_handle* hh, int cls);
  ~ProfScope();
};

// ---------------------------------------------------------------------------
// Device helpers.  All FP64 arithmetic in the parity kernels is compiled
// without FMA contraction so each expression rounds like the Fortran.
__device__ __forceinline__ double dot3(const double a[3], const double b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
__device__ __forceinline__ void cross3(const double x[3], const double y[3], double o[3]) {
  o[0] = x[1] * y[2] - x[2] * y[1];
  o[1] = x[2] * y[0] - x[0] * y[2];
  o[2] = x[0] * y[1] - x[1] * y[0];
}

__device__ __forceinline__ int dg_funijk(const DevParams& p, int i, int j, int k) {
  return j + i * p.c1 + k * p.c2 + p.c3;
}
__device__ __forceinline__ int dg_jof(const DevParams& p, int ijk) {
  return ((ijk - 1) % p.c2) % p.c1 + p.jstart2;
}
__device__ __forceinline__ int dg_iof(const DevParams& p, int ijk) {
  return ((ijk - dg_jof(p, ijk) + p.jstart2 - 1) % p.c2) / p.c1 + p.istart2;
}
__device__ __forceinline__ int dg_kof(const DevParams& p, int ijk) {
  return (ijk - p.c3 - dg_iof(p, ijk) * p.c1 - dg_jof(p, ijk)) / p.c2;
}
// A DES cell as (i, j, k) in one int: 10 bits for i and k, 12 for j (the
// handle set-up checks the grid fits).
constexpr int DG_MAX_IK = 1023, DG_MAX_J = 4095;
__device__ __forceinline__ int pack_ijk(int i, int j, int k) { return i | (j << 10) | (k << 22); }
__device__ __forceinline__ void unpack_ijk(int c, int& i, int& j, int& k) {
  i = c & 1023;
  j = (c >> 10) & 4095;
  k = (c >> 22) & 1023;
}

// Cells of the DES grid, and of the search grid of the pair build, at most
// (with their ghost layers): every cell index and count fits an int.
constexpr long long MAX_GRID_CELLS = 1LL << 28;
// Cells of the search grid of one system when it is finer than its DES grid.
constexpr long long SEARCH_CELLS_CAP = 1LL << 22;

constexpr int MAX_PARTICLES = (1 << 27) - 1;  // particle index in 27 bits of a kept key

__device__ __forceinline__ int dg_ofpos(const DevParams& p, int ax, double x, int start1) {
  return (int)floor((x - p.dg_start[ax]) * p.dg_inv[ax]) + start1;
}

// DESGRID_PIC for one existing particle at x (desgrid_mod.f:877-995): on a
// periodic axis a coordinate whose cell left the domain's cells moves by one
// period (the serial self-exchange of DES_PAR_EXCHANGE,
// mpi_funs_des_mod.f:38-160); then the clamped DES cell.  Returns whether x
// moved.
__device__ __forceinline__ bool dg_place(const DevParams& p, bool per, double4& x, int& cell) {
  bool moved = false;
  if (per) {
    if (p.per[0]) {
      int ci = dg_ofpos(p, 0, x.x, p.istart1);
      if (ci > p.iend1) { x.x = x.x - p.L[0]; moved = true; }
      else if (ci < p.istart1) { x.x = x.x + p.L[0]; moved = true; }
    }
    if (p.per[1]) {
      int cj = dg_ofpos(p, 1, x.y, p.jstart1);
      if (cj > p.jend1) { x.y = x.y - p.L[1]; moved = true; }
      else if (cj < p.jstart1) { x.y = x.y + p.L[1]; moved = true; }
    }
    if (p.per[2] && !p.no_k) {
      int ck = dg_ofpos(p, 2, x.z, p.kstart1);
      if (ck > p.kend1) { x.z = x.z - p.L[2]; moved = true; }
      else if (ck < p.kstart1) { x.z = x.z + p.L[2]; moved = true; }
    }
  }
  int li = min(p.iend2, max(p.istart2, dg_ofpos(p, 0, x.x, p.istart1)));
  int lj = min(p.jend2, max(p.jstart2, dg_ofpos(p, 1, x.y, p.jstart1)));
  int lk = p.no_k ? 1 : min(p.kend2, max(p.kstart2, dg_ofpos(p, 2, x.z, p.kstart1)));
  cell = dg_funijk(p, li, lj, lk);
  return moved;
}

// Minimum-image shift for periodic axes (the copy of j that the reference's
// ghost exchange places next to i).
__device__ __forceinline__ double periodic_shift(const DevParams& p, int ax, double d) {
  if (!p.per[ax]) return 0.0;
  double L = p.L[ax];
  if (d > 0.5 * L) return -L;
  if (d < -0.5 * L) return L;
  return 0.0;
}

// Adds a particle's displacement bound of this step (max(|v|, |v_new|)*dt,
// as float bits rounded up) to the per-step maximum.  Called by every active
// lane of a warp; one atomic per warp, spread over 32 slots.
__device__ __forceinline__ void note_displacement(unsigned* __restrict__ vslot, double disp) {
  const unsigned bits = __float_as_uint(__double2float_ru(disp));
  const unsigned mask = __activemask();
  const unsigned m = __reduce_max_sync(mask, bits);
  const int lane = threadIdx.x & 31;
  if (lane == __ffs(mask) - 1 && m)
    atomicMax(&vslot[((blockIdx.x * blockDim.x + threadIdx.x) >> 5) & 31], m);
}

__device__ __forceinline__ double speed(const double v[3]) {
  return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
}

// Result of the force sum of one particle: either stored into FC/TOW
// (MODE 0) or integrated as CFUPDATEOLD + CFNEWVALUES (cfupdateold.f:33-41,
// cfnewvalues.f:700-812) into the other state buffer (MODE 1 = Euler,
// MODE 2 = Adams-Bashforth).  Velocity updates apply to NORMAL particles,
// position updates to states below NORMAL_GHOST.
// Outputs of DESGRID_PIC when the integration does it for the new positions
// (a null dg_pijk: not done there).
struct CellOut {
  int* dg_pijk = nullptr;
  uint8_t* wall_cand = nullptr;
  const int* fbin_start = nullptr;
  float* wgap = nullptr;  // facet clearance of the last build: -1 (unknown) on a change of cell
};

template <int MODE>
__device__ __forceinline__ void finish_particle(const DevParams& p, int me, int8_t st, const double x[3],
                                                const double v[3], const double w[3], double r, double m,
                                                double omoi, const double f[3], const double t[3],
                                                double4* __restrict__ pos_n, double4* __restrict__ vel_n,
                                                double4* __restrict__ omg_n, double* __restrict__ fc,
                                                double* __restrict__ tow, double* __restrict__ acc_old,
                                                double* __restrict__ rot_acc_old, unsigned* __restrict__ vslot,
                                                CellOut cells = CellOut{}, bool keep_w = false) {
  const size_t n = (size_t)p.n;
  if (MODE == 0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) { fc[c * n + me] = f[c]; tow[c * n + me] = t[c]; }
    return;
  }
  const double dt = p.dt;
  double xn[3], vn[3], wn[3];
  if (MODE == 1) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      vn[c] = v[c];
      if (st == DEM_STATE_NORMAL) vn[c] = v[c] + dt * (f[c] / m + p.grav[c]);
      xn[c] = x[c];
      if (st < DEM_STATE_NORMAL_GHOST) xn[c] = x[c] + vn[c] * dt;
      wn[c] = w[c];
      if (st == DEM_STATE_NORMAL) wn[c] = w[c] + t[c] * omoi * dt;
    }
  } else {
    const bool fp_ok = !(st == DEM_STATE_NONEXISTENT || st == DEM_STATE_ENTERING || st == 102 ||
                         st == DEM_STATE_NORMAL_GHOST || st == 110);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double ao = acc_old[c * n + me], ro = rot_acc_old[c * n + me];
      if (p.first_pass && fp_ok) { ao = f[c] / m + p.grav[c]; ro = t[c]; }
      double a = f[c];
      if (st == DEM_STATE_NORMAL) a = f[c] / m + p.grav[c];
      vn[c] = v[c];
      if (st == DEM_STATE_NORMAL) vn[c] = v[c] + 0.5 * (3.0 * a - ao) * dt;
      acc_old[c * n + me] = a;
      xn[c] = x[c];
      if (st < DEM_STATE_NORMAL_GHOST) xn[c] = x[c] + 0.5 * (v[c] + vn[c]) * dt;
      wn[c] = w[c];
      if (st == DEM_STATE_NORMAL) {
        wn[c] = w[c] + 0.5 * (3.0 * t[c] * omoi - ro) * dt;
        ro = t[c] * omoi;
      }
      rot_acc_old[c * n + me] = ro;
    }
  }
  double4 xo = make_double4(xn[0], xn[1], xn[2], r);
  if (cells.dg_pijk) {
    // the step's DESGRID_PIC for a periodic system, on the new position
    if (st == DEM_STATE_NONEXISTENT) {
      cells.dg_pijk[me] = 0;
      cells.wall_cand[me] = 0;
    } else {
      int c;
      dg_place(p, true, xo, c);
      if (cells.dg_pijk[me] != c) cells.wgap[me] = -1.0f;
      cells.dg_pijk[me] = c;
      const int fc = p.cell_off + c - 1;
      cells.wall_cand[me] = cells.fbin_start[fc + 1] > cells.fbin_start[fc] ? 1 : 0;
    }
  }
  pos_n[me] = xo;
  vel_n[me] = make_double4(vn[0], vn[1], vn[2], m);
  // keep_w: the spin stays as it is (the gather did not read it)
  if (!keep_w) omg_n[me] = make_double4(wn[0], wn[1], wn[2], omoi);
  // |x_new - x| <= max(|v|, |v_new|) * dt for both integrators
  note_displacement(vslot, st < DEM_STATE_NORMAL_GHOST ? fmax(speed(v), speed(vn)) * dt : 0.0);
}

}  // namespace demb

#define DEM_LAUNCH(h) ((h)->launches++)

namespace demb {
// A single handle with a periodic axis places its particles in their DES
// cells in the integrating gather (the step's DESGRID_PIC then runs only on
// neighbour-search steps, where it repeats the same placement).
inline bool cells_in_gather(const dem_handle* h) {
  const DevParams& p = h->dp;
  // not with flow boundaries: their cell tests read the cells of the last
  // DESGRID_PIC, which the placement would move ahead
  return !h->batch() && h->obc.empty() && h->ibc.empty() && (p.per[0] || p.per[1] || (p.per[2] && !p.no_k));
}
template <int MODE, bool B>
inline CellOut gather_cells(const dem_handle* h) {
  CellOut c;
  if (MODE != 0 && !B && cells_in_gather(h)) {
    c.dg_pijk = h->dg_pijk;
    c.wall_cand = h->wall_cand;
    c.fbin_start = h->fbin_start;
    c.wgap = h->wgap;
  }
  return c;
}
}  // namespace demb
