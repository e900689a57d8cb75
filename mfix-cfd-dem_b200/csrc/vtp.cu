// vtp.cu -- particle output as VTK PolyData (.vtp), the file WRITE_VTP_FILE
// writes for a VTK region of particle data (model/des/vtp_mod.f:705-1257).
//
// Layout as OPEN_VTP_FILE_BIN, WRITE_GEOMETRY_IN_VTP_BIN,
// WRITE_SCALAR_IN_VTP_BIN / WRITE_VECTOR_IN_VTP_BIN and CLOSE_VTP_FILE_BIN
// produce it (vtp_mod.f:1540-2906): an XML header (byte_order="BigEndian"),
// one Piece with NumberOfPoints, the Points DataArray "coordinates" and the
// PointData arrays "Diameter" and "Velocity" (and "Angular_velocity" when
// asked) as Float32 with format="appended", then <AppendedData
// encoding="raw">, an underscore and, for every array in the same order, a
// 4-byte length followed by the big-endian Float32 values.  The offset of an
// array is the byte count of the arrays before it, their lengths included.
//
// The particles written are those of the region, as
// SETUP_VTK_REGION_PARTICLES selects them (vtp_mod.f:2925-3172): NORMAL (or
// RIGID) particles of the region's phases whose centre is inside the box
// ('C'), which lie entirely inside it ('P') or which intersect it ('I');
// slices (VTK_NXS...) are not built.  Host code only: the state comes from
// the device through dem_download_state.
#include "dem_internal.cuh"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace demb;

namespace {

inline uint32_t be32f(float v) {
  uint32_t u;
  memcpy(&u, &v, 4);
  return __builtin_bswap32(u);
}

bool keep(const dem_vtp_options* o, const double x[3], double r) {
  if (!o || !o->use_box) return true;
  for (int c = 0; c < 3; ++c) {
    const double lo = o->box_lo[c], hi = o->box_hi[c];
    bool in;
    switch (o->select_mode) {
      case 'P': in = lo <= x[c] - r && x[c] + r <= hi; break;
      case 'I': in = !(hi <= x[c] - r || x[c] + r <= lo); break;
      default: in = lo <= x[c] && x[c] <= hi; break;  // 'C'
    }
    if (!in) return false;
  }
  return true;
}

}  // namespace

extern "C" {

int dem_vtp_write(const char* path, const dem_vtp_options* opt, int32_t max_pip, const double* pos,
                  const double* vel, const double* omega, const double* radius, const int8_t* state,
                  const int32_t* phase, int64_t* n_written) {
  if (!path || max_pip < 0 || !pos || !vel || !radius || !state) return DEM_ERR_ARG;
  const bool ang = opt && opt->angular_velocity;
  if (ang && !omega) return DEM_ERR_ARG;
  if (opt && opt->use_box && opt->select_mode != 'C' && opt->select_mode != 'P' && opt->select_mode != 'I' &&
      opt->select_mode != 0)
    return DEM_ERR_ARG;
  const size_t n = (size_t)max_pip;
  std::vector<int> sel;
  for (size_t l = 0; l < n; ++l) {
    if (state[l] != DEM_STATE_NORMAL && state[l] != DEM_STATE_RIGID) continue;
    if (opt && opt->phase_mask && phase) {
      const int m = phase[l];
      if (m < 1 || m > 32 || !((opt->phase_mask >> (m - 1)) & 1u)) continue;
    }
    const double x[3] = {pos[l], pos[n + l], pos[2 * n + l]};
    if (keep(opt, x, radius[l])) sel.push_back((int)l);
  }
  const long long np = (long long)sel.size();
  if (np > INT32_MAX / 12) return DEM_ERR_CAPACITY;
  const int nb_vec = (int)(np * 3 * 4), nb_sca = (int)(np * 4);
  FILE* f = fopen(path, "wb");
  if (!f) return DEM_ERR_ARG;
  std::string h;
  char line[512];
  h += "<?xml version=\"1.0\"?>\n";
  snprintf(line, sizeof line, "<!-- Time = %.17g sec. -->\n", opt ? opt->time : 0.0);
  h += line;
  h += "<VTKFile type=\"PolyData\" version=\"0.1\" byte_order=\"BigEndian\">\n";
  h += "  <PolyData>\n";
  snprintf(line, sizeof line,
           "    <Piece NumberOfPoints=\"%lld\" NumberOfVerts=\"0\" NumberOfLines=\"0\" NumberOfStrips=\"0\" "
           "NumberOfPolys=\"0\">\n", np);
  h += line;
  h += "      <Points>\n";
  h += "        <DataArray type=\"Float32\" Name=\"coordinates\" NumberOfComponents=\"3\" format=\"appended\" "
       "offset=\"0\" />\n";
  h += "      </Points>\n";
  h += "      <PointData Scalars=\"Diameter\" Vectors=\"Velocity\">\n";
  long long off = 4 + (long long)nb_vec;
  snprintf(line, sizeof line,
           "        <DataArray type=\"Float32\" Name=\"Diameter\" format=\"appended\" offset=\"%lld\" />\n", off);
  h += line;
  off += 4 + nb_sca;
  snprintf(line, sizeof line,
           "        <DataArray type=\"Float32\" Name=\"Velocity\" NumberOfComponents=\"3\" format=\"appended\" "
           "offset=\"%lld\" />\n", off);
  h += line;
  off += 4 + nb_vec;
  if (ang) {
    snprintf(line, sizeof line,
             "        <DataArray type=\"Float32\" Name=\"Angular_velocity\" NumberOfComponents=\"3\" "
             "format=\"appended\" offset=\"%lld\" />\n", off);
    h += line;
  }
  h += "      </PointData>\n";
  h += "      <Verts> </Verts>\n      <Lines> </Lines>\n      <Strips> </Strips>\n      <Polys> </Polys>\n";
  h += "    </Piece>\n  </PolyData>\n  <AppendedData encoding=\"raw\">\n_";
  bool ok = fwrite(h.data(), 1, h.size(), f) == h.size();
  std::vector<uint32_t> buf;
  auto put_len = [&](int nbytes) {
    const uint32_t b = __builtin_bswap32((uint32_t)nbytes);
    ok = ok && fwrite(&b, 4, 1, f) == 1;
  };
  auto put_vec = [&](const double* a) {
    put_len(nb_vec);
    buf.resize((size_t)np * 3);
    for (long long k = 0; k < np; ++k)
      for (int c = 0; c < 3; ++c) buf[3 * k + c] = be32f((float)a[c * n + sel[k]]);
    ok = ok && fwrite(buf.data(), 4, buf.size(), f) == buf.size();
  };
  put_vec(pos);
  put_len(nb_sca);
  buf.resize((size_t)np);
  for (long long k = 0; k < np; ++k) buf[k] = be32f((float)(2.0 * radius[sel[k]]));
  ok = ok && fwrite(buf.data(), 4, buf.size(), f) == buf.size();
  put_vec(vel);
  if (ang) put_vec(omega);
  const char* tail = "\n  </AppendedData>\n</VTKFile>\n";
  ok = ok && fwrite(tail, 1, strlen(tail), f) == strlen(tail);
  if (fclose(f) != 0) ok = false;
  if (!ok) return DEM_ERR_ARG;
  if (n_written) *n_written = np;
  return 0;
}

int dem_write_vtp(dem_handle* h, const char* path, const dem_vtp_options* opt, int64_t* n_written) {
  if (!h) return DEM_ERR_ARG;
  cudaSetDevice(h->dev);
  if (h->batch()) return set_err(h, DEM_ERR_ARG, "particle output is per system; not available on a batch handle");
  if (!h->have_state) return set_err(h, DEM_ERR_STATE, "no particle state uploaded");
  const size_t n = (size_t)h->n;
  std::vector<double> pos(3 * n), vel(3 * n), omega(3 * n), radius(n);
  std::vector<int8_t> state(n);
  if (int rc = dem_download_state(h, pos.data(), vel.data(), omega.data(), state.data(), h->n)) return rc;
  std::vector<double4> p4(n);
  std::vector<uint8_t> ph(n);
  cudaMemcpyAsync(p4.data(), h->pos4[h->cur], sizeof(double4) * n, cudaMemcpyDeviceToHost, h->stream);
  cudaMemcpyAsync(ph.data(), h->phase, n, cudaMemcpyDeviceToHost, h->stream);
  if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "vtp write")) return rc;
  std::vector<int32_t> phase(n);
  for (size_t l = 0; l < n; ++l) { radius[l] = p4[l].w; phase[l] = (int32_t)ph[l] + 1; }
  const int rc = dem_vtp_write(path, opt, h->n, pos.data(), vel.data(), omega.data(), radius.data(), state.data(),
                               phase.data(), n_written);
  if (rc) return set_err(h, rc, "particle output write failed");
  return 0;
}

}  // extern "C"
