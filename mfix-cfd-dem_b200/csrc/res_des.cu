// res_des.cu -- DEM restart file (RES) writer and reader.
//
// The file layout is the one WRITE_RES0_DES / READ_RES0_DES use for a serial
// run (model/des/write_res0_des.f:44-208, read_res0_des.f, record writers in
// write_res1_des_mod.f and out_bin_512.f / out_bin_512i.f):
//
//   * direct-access records of OPEN_N1 = 512 bytes (machine_mod.f:8), values
//     big-endian (the build compiles Fortran with -fconvert=big-endian,
//     CMakeLists.txt:264-266), INTEGER 4 bytes, DOUBLE PRECISION 8 bytes;
//   * a scalar takes one record; an array of N values takes ceil(N/64)
//     records of doubles or ceil(N/128) records of integers, and one record
//     when N = 0 (OUT_BIN_512: N <= NWORDS writes one record);
//   * record order: VERSION, particle count, ghost count (0), pair count;
//     VTP_FINDEX, TECPLOT_FINDEX, DTSOLID; DES_POS_NEW (lDIMN columns);
//     iGLOBAL_ID; PARTICLE_STATE; DES_VEL_NEW (lDIMN); OMEGA_NEW (column 1
//     in 2D, all three in 3D); DES_RADIUS; RO_SOL; PIJK(:,5);
//     DES_USR_VAR_SIZE (0); RESIDENCE_TIME; NEIGHBORS; NEIGHBOR_INDEX;
//     PFT_NEIGHBOR (lDIMN components); DEM_BCMI (0).
//
// Particle arrays hold the existing non-ghost particles in slot order (the
// packing of DES_GATHER, mpi_comm_des_mod.f:222-247); a particle's global id
// is its 1-based slot.  Pair arrays hold the entries whose two particles
// exist, in NEIGHBORS order (WRITE_RES_cARRAY, write_res1_des_mod.f).  Two
// deliberate differences from the reference writer, both in the pair section:
// the owner filter uses the true owner of each entry (the reference's running
// `part` counter lags behind after an empty row), and the second pair array
// holds the global id of each entry's owner, where the reference writes
// iGLOBAL_ID(NEIGHBOR_INDEX(LC)), an index into a per-particle array by a pair
// position that its reader does not use (GLOBAL_TO_LOC_COL,
// read_res1_des_mod.f:437-474, matches nothing).  With the owners in the
// file the reader here restores the pair list and its tangential history
// exactly; for a file written by the reference, pass restore_pairs = 0 and
// rebuild the list from the positions, which is what the reference's own
// serial restart amounts to.  Wall-contact and Adams-Bashforth histories are
// not in the format (nor restored by the reference).
#include "dem_internal.cuh"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

using namespace demb;

namespace {

constexpr int REC = 512;
constexpr int NW_DP = REC / 8;   // NWORDS_DP
constexpr int NW_I = REC / 4;    // NWORDS_I

// VERSION = 1.2 in write_res0_des.f is a default-real literal stored in a
// double: the file holds the single-precision value widened.
const double RES_VERSION = (double)1.2f;

inline uint32_t be32(uint32_t v) { return __builtin_bswap32(v); }
inline uint64_t be64(uint64_t v) { return __builtin_bswap64(v); }

struct RecFile {
  FILE* f = nullptr;
  long next = 1;  // 1-based record number
  unsigned char buf[REC];
  bool ok = true;

  void put_record(const void* data, size_t bytes) {
    memset(buf, 0, REC);
    memcpy(buf, data, bytes);
    if (fseek(f, (next - 1) * (long)REC, SEEK_SET) != 0 || fwrite(buf, 1, REC, f) != (size_t)REC) ok = false;
    ++next;
  }
  bool get_record() {
    if (fseek(f, (next - 1) * (long)REC, SEEK_SET) != 0 || fread(buf, 1, REC, f) != (size_t)REC) ok = false;
    ++next;
    return ok;
  }
  void put_i(int32_t v) {
    const uint32_t b = be32((uint32_t)v);
    put_record(&b, 4);
  }
  void put_d(double v) {
    uint64_t u;
    memcpy(&u, &v, 8);
    u = be64(u);
    put_record(&u, 8);
  }
  template <class Get>
  void put_di(int64_t n, Get get) {  // doubles
    int64_t i = 0;
    do {
      const int64_t m = n - i < NW_DP ? n - i : NW_DP;
      uint64_t w[NW_DP];
      for (int64_t k = 0; k < m; ++k) {
        const double v = get(i + k);
        memcpy(&w[k], &v, 8);
        w[k] = be64(w[k]);
      }
      put_record(w, 8 * (size_t)m);
      i += m;
    } while (i < n);
  }
  template <class Get>
  void put_ii(int64_t n, Get get) {  // integers
    int64_t i = 0;
    do {
      const int64_t m = n - i < NW_I ? n - i : NW_I;
      uint32_t w[NW_I];
      for (int64_t k = 0; k < m; ++k) w[k] = be32((uint32_t)get(i + k));
      put_record(w, 4 * (size_t)m);
      i += m;
    } while (i < n);
  }
  int32_t get_i() {
    get_record();
    uint32_t b;
    memcpy(&b, buf, 4);
    return (int32_t)be32(b);
  }
  double get_d() {
    get_record();
    uint64_t u;
    memcpy(&u, buf, 8);
    u = be64(u);
    double v;
    memcpy(&v, &u, 8);
    return v;
  }
  template <class Set>
  void get_di(int64_t n, Set set) {
    int64_t i = 0;
    do {
      const int64_t m = n - i < NW_DP ? n - i : NW_DP;
      if (!get_record()) return;
      for (int64_t k = 0; k < m; ++k) {
        uint64_t u;
        memcpy(&u, buf + 8 * k, 8);
        u = be64(u);
        double v;
        memcpy(&v, &u, 8);
        set(i + k, v);
      }
      i += m;
    } while (i < n);
  }
  template <class Set>
  void get_ii(int64_t n, Set set) {
    int64_t i = 0;
    do {
      const int64_t m = n - i < NW_I ? n - i : NW_I;
      if (!get_record()) return;
      for (int64_t k = 0; k < m; ++k) {
        uint32_t b;
        memcpy(&b, buf + 4 * k, 4);
        set(i + k, (int32_t)be32(b));
      }
      i += m;
    } while (i < n);
  }
};

inline bool exists(int8_t s) { return s != DEM_STATE_NONEXISTENT && s < DEM_STATE_NORMAL_GHOST; }

}  // namespace

extern "C" {

static int res_write(const char* path, const dem_res_info* info, int32_t max_pip, int32_t no_k, const double* pos,
                     const double* vel, const double* omega, const double* radius, const int8_t* state,
                     const int32_t* phase, const int32_t* neighbor_index, const int32_t* neighbors, const double* pft,
                     int64_t n_pairs, const std::vector<dem_handle::Inflow>* mi) {
  if (!path || !info || max_pip < 0 || !pos || !vel || !omega || !radius || !state || !phase) return DEM_ERR_ARG;
  if (n_pairs < 0 || (n_pairs > 0 && (!neighbor_index || !neighbors || !pft))) return DEM_ERR_ARG;
  const int dimn = no_k ? 2 : 3;
  const size_t n = (size_t)max_pip;
  std::vector<int> slot;  // packed particle -> slot
  std::vector<int> gid(n, 0);
  for (size_t l = 0; l < n; ++l)
    if (exists(state[l])) { slot.push_back((int)l); gid[l] = (int)l + 1; }
  for (int32_t l = 0; l < max_pip; ++l)
    if (exists(state[l]) && (phase[l] < 1 || phase[l] > DEM_MAX_PHASES)) return DEM_ERR_ARG;
  // pair entries whose two particles exist, with their owners
  std::vector<int64_t> keep;
  std::vector<int> owner;
  {
    int64_t s = 0;
    for (int32_t i = 0; i < max_pip; ++i) {
      const int64_t e = neighbor_index ? (int64_t)neighbor_index[i] - 1 : 0;
      if (e < s || e > n_pairs) return DEM_ERR_ARG;
      for (int64_t c = s; c < e; ++c) {
        const int j = neighbors[c] - 1;
        if (j < 0 || j >= max_pip) return DEM_ERR_ARG;
        if (exists(state[i]) && exists(state[j])) { keep.push_back(c); owner.push_back(i); }
      }
      s = e;
    }
  }
  const int64_t np = (int64_t)slot.size(), nc = (int64_t)keep.size();
  if (np > INT32_MAX || nc > INT32_MAX) return DEM_ERR_CAPACITY;
  RecFile w;
  w.f = fopen(path, "wb");
  if (!w.f) return DEM_ERR_ARG;
  // INIT_WRITE_RES_DES
  w.put_d(RES_VERSION);
  w.put_i((int32_t)np);
  w.put_i(0);
  w.put_i((int32_t)nc);
  w.put_i(info->vtp_findex);
  w.put_i(info->tecplot_findex);
  w.put_d(info->dtsolid);
  for (int c = 0; c < dimn; ++c) w.put_di(np, [&](int64_t k) { return pos[c * n + slot[k]]; });
  w.put_ii(np, [&](int64_t k) { return gid[slot[k]]; });
  w.put_ii(np, [&](int64_t k) { return (int32_t)state[slot[k]]; });
  for (int c = 0; c < dimn; ++c) w.put_di(np, [&](int64_t k) { return vel[c * n + slot[k]]; });
  for (int c = 0; c < (no_k ? 1 : 3); ++c) w.put_di(np, [&](int64_t k) { return omega[c * n + slot[k]]; });
  w.put_di(np, [&](int64_t k) { return radius[slot[k]]; });
  w.put_di(np, [&](int64_t k) { return info->ro_sol[phase[slot[k]] - 1]; });
  w.put_ii(np, [&](int64_t k) { return phase[slot[k]]; });
  w.put_i(0);                                      // DES_USR_VAR_SIZE
  w.put_di(np, [&](int64_t) { return 0.0; });      // RESIDENCE_TIME
  w.put_ii(nc, [&](int64_t k) { return gid[neighbors[keep[k]] - 1]; });
  w.put_ii(nc, [&](int64_t k) { return gid[owner[k]]; });
  for (int c = 0; c < dimn; ++c) w.put_di(nc, [&](int64_t k) { return pft[3 * keep[k] + c]; });
  // DEM_BCMI, then per boundary DEM_MI_TIME and DEM_MI's VACANCY, OCCUPANTS,
  // WINDOW, OFFSET, L, W, H, P, Q (write_res0_des.f:197-210)
  const int32_t nbc = mi ? (int32_t)mi->size() : 0;
  w.put_i(nbc);
  for (int32_t b = 0; b < nbc; ++b) {
    const dem_handle::Inflow& I = (*mi)[b];
    const int32_t occ = (int32_t)I.p.size();
    w.put_d(I.bc.mi_time);
    w.put_i(I.bc.vacancy);
    w.put_i(occ);
    w.put_d(I.bc.window);
    w.put_d(I.bc.offset);
    w.put_i(I.bc.l_index);
    w.put_ii(occ, [&](int64_t k) { return I.w[k]; });
    w.put_ii(occ, [&](int64_t k) { return I.hh[k]; });
    w.put_di(occ, [&](int64_t k) { return I.p[k]; });
    w.put_di(occ, [&](int64_t k) { return I.q[k]; });
  }
  const bool ok = w.ok;
  if (fclose(w.f) != 0 || !ok) return DEM_ERR_ARG;
  return 0;
}

int dem_res_read(const char* path, dem_res_info* info, int32_t max_pip, int32_t no_k, double* pos, double* vel,
                 double* omega, double* radius, double* ro_sol, int8_t* state, int32_t* phase,
                 int32_t* pair_owner, int32_t* pair_neighbor, double* pft, int64_t pair_cap) {
  if (!path || !info) return DEM_ERR_ARG;
  const int dimn = no_k ? 2 : 3;
  RecFile r;
  r.f = fopen(path, "rb");
  if (!r.f) return DEM_ERR_ARG;
  struct Closer { FILE* f; ~Closer() { fclose(f); } } closer{r.f};
  const double version = r.get_d();
  const int32_t np = r.get_i();
  r.get_i();  // ghosts
  const int32_t nc = r.get_i();
  if (!r.ok || np < 0 || nc < 0) return DEM_ERR_ARG;
  info->version = version;
  info->n_particles = np;
  info->n_pairs = nc;
  if (!pos) return 0;  // header only
  if (!(version >= RES_VERSION)) return DEM_ERR_ARG;  // PIJK(:,5) is stored from version 1.2
  if (np > max_pip || !vel || !omega || !radius || !ro_sol || !state || !phase) return DEM_ERR_ARG;
  if (pair_owner && (pair_cap < nc || !pair_neighbor || !pft)) return DEM_ERR_CAPACITY;
  const size_t n = (size_t)max_pip;
  for (size_t l = 0; l < n; ++l) {
    state[l] = DEM_STATE_NONEXISTENT;
    radius[l] = 0.0; ro_sol[l] = 0.0; phase[l] = 1;
    for (int c = 0; c < 3; ++c) { pos[c * n + l] = 0.0; vel[c * n + l] = 0.0; omega[c * n + l] = 0.0; }
  }
  info->vtp_findex = r.get_i();
  info->tecplot_findex = r.get_i();
  info->dtsolid = r.get_d();
  for (int c = 0; c < dimn; ++c) r.get_di(np, [&](int64_t k, double v) { pos[c * n + k] = v; });
  std::vector<int32_t> gid(np);
  r.get_ii(np, [&](int64_t k, int32_t v) { gid[k] = v; });
  r.get_ii(np, [&](int64_t k, int32_t v) { state[k] = (int8_t)v; });
  for (int c = 0; c < dimn; ++c) r.get_di(np, [&](int64_t k, double v) { vel[c * n + k] = v; });
  for (int c = 0; c < (no_k ? 1 : 3); ++c) r.get_di(np, [&](int64_t k, double v) { omega[c * n + k] = v; });
  r.get_di(np, [&](int64_t k, double v) { radius[k] = v; });
  r.get_di(np, [&](int64_t k, double v) { ro_sol[k] = v; });
  r.get_ii(np, [&](int64_t k, int32_t v) { phase[k] = v; });
  const int32_t nusr = r.get_i();
  if (!r.ok || nusr < 0) return DEM_ERR_ARG;
  for (int32_t u = 0; u < nusr; ++u) r.get_di(np, [](int64_t, double) {});   // DES_USR_VAR
  r.get_di(np, [](int64_t, double) {});                                       // RESIDENCE_TIME
  if (!r.ok) return DEM_ERR_ARG;
  if (!pair_owner) return 0;
  // global id -> packed slot
  int32_t maxid = 0;
  for (int32_t v : gid) maxid = v > maxid ? v : maxid;
  std::vector<int32_t> local((size_t)maxid + 1, 0);
  for (int32_t k = 0; k < np; ++k) {
    if (gid[k] < 1) return DEM_ERR_ARG;
    local[gid[k]] = k + 1;
  }
  auto to_local = [&](int32_t g) { return (g >= 1 && g <= maxid) ? local[g] : 0; };
  bool bad = false;
  r.get_ii(nc, [&](int64_t k, int32_t v) { pair_neighbor[k] = to_local(v); bad = bad || !pair_neighbor[k]; });
  r.get_ii(nc, [&](int64_t k, int32_t v) { pair_owner[k] = to_local(v); bad = bad || !pair_owner[k]; });
  for (int c = 0; c < 3; ++c)
    for (int64_t k = 0; k < nc; ++k) pft[3 * k + c] = 0.0;
  for (int c = 0; c < dimn; ++c) r.get_di(nc, [&](int64_t k, double v) { pft[3 * k + c] = v; });
  if (!r.ok) return DEM_ERR_ARG;
  return bad ? DEM_ERR_STATE : 0;
}

int dem_res_write(const char* path, const dem_res_info* info, int32_t max_pip, int32_t no_k, const double* pos,
                  const double* vel, const double* omega, const double* radius, const int8_t* state,
                  const int32_t* phase, const int32_t* neighbor_index, const int32_t* neighbors, const double* pft,
                  int64_t n_pairs) {
  return res_write(path, info, max_pip, no_k, pos, vel, omega, radius, state, phase, neighbor_index, neighbors, pft,
                   n_pairs, nullptr);
}

int dem_res_read_inflow(const char* path, int32_t no_k, int32_t* n_bc, dem_res_inflow* mi, int32_t max_bc,
                        int32_t* wc, int32_t* hc, double* pc, double* qc, int32_t max_occ) {
  if (!path || !n_bc || max_bc < 0 || (max_bc > 0 && !mi) || max_occ < 0) return DEM_ERR_ARG;
  const int dimn = no_k ? 2 : 3;
  RecFile r;
  r.f = fopen(path, "rb");
  if (!r.f) return DEM_ERR_ARG;
  struct Closer { FILE* f; ~Closer() { fclose(f); } } closer{r.f};
  r.get_d();
  const int32_t np = r.get_i();
  r.get_i();
  const int32_t nc = r.get_i();
  if (!r.ok || np < 0 || nc < 0) return DEM_ERR_ARG;
  // skip the particle and pair sections record by record
  auto skip_d = [&](int64_t m) { r.get_di(m, [](int64_t, double) {}); };
  auto skip_i = [&](int64_t m) { r.get_ii(m, [](int64_t, int32_t) {}); };
  r.get_i(); r.get_i(); r.get_d();
  for (int c = 0; c < dimn; ++c) skip_d(np);
  skip_i(np); skip_i(np);
  for (int c = 0; c < dimn; ++c) skip_d(np);
  for (int c = 0; c < (no_k ? 1 : 3); ++c) skip_d(np);
  skip_d(np); skip_d(np); skip_i(np);
  const int32_t nusr = r.get_i();
  if (!r.ok || nusr < 0) return DEM_ERR_ARG;
  for (int32_t u = 0; u < nusr; ++u) skip_d(np);
  skip_d(np);
  skip_i(nc); skip_i(nc);
  for (int c = 0; c < dimn; ++c) skip_d(nc);
  const int32_t nbc = r.get_i();
  if (!r.ok || nbc < 0) return DEM_ERR_ARG;
  *n_bc = nbc;
  for (int32_t b = 0; b < nbc; ++b) {
    dem_res_inflow rec{};
    rec.mi_time = r.get_d();
    rec.vacancy = r.get_i();
    rec.occupants = r.get_i();
    rec.window = r.get_d();
    rec.offset = r.get_d();
    rec.l_index = r.get_i();
    if (!r.ok || rec.occupants < 0) return DEM_ERR_ARG;
    const int32_t occ = rec.occupants;
    const bool keep = b < max_bc;
    if (keep) mi[b] = rec;
    if (keep && (wc || hc || pc || qc) && occ > max_occ) return DEM_ERR_CAPACITY;
    const size_t row = (size_t)b * (size_t)max_occ;
    r.get_ii(occ, [&](int64_t k, int32_t v) { if (keep && wc) wc[row + k] = v; });
    r.get_ii(occ, [&](int64_t k, int32_t v) { if (keep && hc) hc[row + k] = v; });
    r.get_di(occ, [&](int64_t k, double v) { if (keep && pc) pc[row + k] = v; });
    r.get_di(occ, [&](int64_t k, double v) { if (keep && qc) qc[row + k] = v; });
    if (!r.ok) return DEM_ERR_ARG;
  }
  return 0;
}

int dem_write_res0_des(dem_handle* h, const char* path, const dem_res_info* info) {
  if (!h) return DEM_ERR_ARG;
  cudaSetDevice(h->dev);
  if (h->batch()) return set_err(h, DEM_ERR_ARG, "restart files are per system; not available on a batch handle");
  if (!path || !info) return set_err(h, DEM_ERR_ARG, "null argument");
  if (!h->have_state) return set_err(h, DEM_ERR_STATE, "no particle state uploaded");
  const size_t n = (size_t)h->n;
  std::vector<double> pos(3 * n), vel(3 * n), omega(3 * n), radius(n);
  std::vector<int8_t> state(n);
  if (int rc = dem_download_state(h, pos.data(), vel.data(), omega.data(), state.data(), h->n)) return rc;
  std::vector<double4> p4(n);
  std::vector<uint8_t> ph(n);
  cudaMemcpyAsync(p4.data(), h->pos4[h->cur], sizeof(double4) * n, cudaMemcpyDeviceToHost, h->stream);
  cudaMemcpyAsync(ph.data(), h->phase, n, cudaMemcpyDeviceToHost, h->stream);
  if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "restart write")) return rc;
  std::vector<int32_t> phase(n);
  for (size_t l = 0; l < n; ++l) { radius[l] = p4[l].w; phase[l] = (int32_t)ph[l] + 1; }
  std::vector<int32_t> ni(n), nb;
  std::vector<double> pf;
  int64_t P = 0;
  if (h->have_pairs) {
    if (int rc = dem_pair_count(h, &P)) return rc;
    nb.resize((size_t)(P ? P : 1));
    pf.resize(3 * (size_t)(P ? P : 1));
    if (int rc = dem_download_pairs(h, ni.data(), nb.data(), pf.data(), P ? P : 1, h->n)) return rc;
  }
  const int rc = res_write(path, info, h->n, h->dp.no_k, pos.data(), vel.data(), omega.data(), radius.data(),
                           state.data(), phase.data(), P ? ni.data() : nullptr, P ? nb.data() : nullptr,
                           P ? pf.data() : nullptr, P, &h->ibc);
  if (rc) return set_err(h, rc, "restart file write failed");
  return 0;
}

int dem_read_res0_des(dem_handle* h, const char* path, int32_t restore_pairs, dem_res_info* info) {
  if (!h) return DEM_ERR_ARG;
  cudaSetDevice(h->dev);
  if (h->batch()) return set_err(h, DEM_ERR_ARG, "restart files are per system; not available on a batch handle");
  if (!path || !info) return set_err(h, DEM_ERR_ARG, "null argument");
  dem_res_info hd{};
  if (int rc = dem_res_read(path, &hd, 0, h->dp.no_k, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                            nullptr, nullptr, nullptr, nullptr, 0))
    return set_err(h, rc, "cannot read restart file header");
  if (hd.n_particles > h->n) return set_err(h, DEM_ERR_CAPACITY, "restart file holds more particles than max_pip");
  const size_t n = (size_t)h->n, P = (size_t)hd.n_pairs;
  std::vector<double> pos(3 * n), vel(3 * n), omega(3 * n), radius(n), ro(n), pmass(n), omoi(n);
  std::vector<int8_t> state(n);
  std::vector<int32_t> phase(n), own(P ? P : 1), nbr(P ? P : 1);
  std::vector<double> pft(3 * (P ? P : 1));
  int rc = dem_res_read(path, info, h->n, h->dp.no_k, pos.data(), vel.data(), omega.data(), radius.data(),
                        ro.data(), state.data(), phase.data(), restore_pairs ? own.data() : nullptr,
                        nbr.data(), pft.data(), (int64_t)(P ? P : 1));
  if (rc) return set_err(h, rc, "restart file read failed");
  // PVOL, PMASS, OMOI of a sphere (make_arrays_des.f:287-291), with R**3 as
  // x*(x*x) (the reference's pow wrapper for an integral exponent)
  const double pi = 4.0 * std::atan(1.0);
  for (size_t l = 0; l < n; ++l) {
    if (state[l] == DEM_STATE_NONEXISTENT) { pmass[l] = 0.0; omoi[l] = 0.0; continue; }
    const double r = radius[l];
    const double pvol = ((4.0 / 3.0) * pi) * (r * (r * r));
    pmass[l] = pvol * ro[l];
    omoi[l] = 2.5 / (pmass[l] * (r * r));
  }
  // DEM_MI_TIME and VACANCY of the installed inflow boundaries come from the
  // file (read_res0_des.f:205-221).  The boundaries' layout is installed by
  // the caller, so the file must hold the same boundaries: as many, each
  // with the same OCCUPANTS and the same seeding offsets P and Q.  Checked
  // before anything is uploaded.
  const size_t nbi = h->ibc.size();
  std::vector<dem_res_inflow> mi(nbi ? nbi : 1);
  if (nbi) {
    int32_t mocc = 1;
    for (const auto& I : h->ibc) mocc = std::max<int32_t>(mocc, I.bc.occupants);
    std::vector<double> fp(nbi * (size_t)mocc), fq(nbi * (size_t)mocc);
    int32_t nbc = 0;
    const int rr = dem_res_read_inflow(path, h->dp.no_k, &nbc, mi.data(), (int32_t)nbi, nullptr, nullptr,
                                       fp.data(), fq.data(), mocc);
    if (rr == DEM_ERR_CAPACITY)
      return set_err(h, DEM_ERR_ARG, "inflow layout in the restart file differs from the installed one");
    if (rr) return set_err(h, DEM_ERR_STATE, "restart file has no readable mass-inflow section");
    if (nbc != (int32_t)nbi) {
      char b[160];
      snprintf(b, sizeof b, "restart file holds %d mass-inflow boundaries, the handle has %zu", nbc, nbi);
      return set_err(h, DEM_ERR_STATE, b);
    }
    for (size_t b = 0; b < nbi; ++b) {
      const auto& I = h->ibc[b];
      bool same = mi[b].occupants == I.bc.occupants && mi[b].vacancy >= 1 &&
                  !(mi[b].occupants > 0 && mi[b].vacancy > mi[b].occupants);
      for (int k = 0; same && k < I.bc.occupants; ++k)
        same = fp[b * (size_t)mocc + k] == I.p[k] && fq[b * (size_t)mocc + k] == I.q[k];
      if (!same) return set_err(h, DEM_ERR_ARG, "inflow layout in the restart file differs from the installed one");
    }
  }
  if ((rc = dem_upload_state(h, pos.data(), vel.data(), omega.data(), radius.data(), pmass.data(), omoi.data(),
                             state.data(), phase.data(), h->n)))
    return rc;
  for (size_t b = 0; b < nbi; ++b) {
    h->ibc[b].bc.vacancy = mi[b].vacancy;
    h->ibc[b].bc.mi_time = mi[b].mi_time;
  }
  if (!restore_pairs) return 0;
  // entries grouped by owner in the file's order -> CSR with 1-based ends
  std::vector<int32_t> ni(n, 0);
  std::vector<int64_t> cnt(n + 1, 0);
  for (size_t k = 0; k < P; ++k) cnt[own[k]]++;  // own is 1-based
  for (size_t i = 1; i <= n; ++i) cnt[i] += cnt[i - 1];
  std::vector<int64_t> at(cnt.begin(), cnt.end() - 1);
  std::vector<int32_t> nb(P ? P : 1);
  std::vector<double> pf(3 * (P ? P : 1));
  for (size_t k = 0; k < P; ++k) {
    const int64_t q = at[own[k] - 1]++;
    nb[q] = nbr[k];
    for (int c = 0; c < 3; ++c) pf[3 * q + c] = pft[3 * k + c];
  }
  for (size_t i = 0; i < n; ++i) ni[i] = (int32_t)cnt[i + 1] + 1;
  return dem_upload_pairs(h, ni.data(), nb.data(), pf.data(), (int64_t)P, h->n);
}

}  // extern "C"
