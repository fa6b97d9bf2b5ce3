// Host-side input: the recon-parameter YAML file and the FreeCT 2-file scan
// format (no GPU involved).
//
// Recon YAML: the flat key list parse_config reads
// (applications/fct_wfbp/src/parse_config.cpp:31-63). FreeCT scan:
// <dir>/meta.yaml written by RawDataSet::getYAMLEmitter
// (modules/fct_read/src/RawDataSet.cpp:17-45) and <dir>/projections.dat,
// frames of {float angle, axial, radial; float data[rows][channels]}
// (RawDataSet.cpp:96-104, FreeCTFrame::readFromFile,
// FreeCTDataSet.cpp:8-21). The frame stride is fixed, so any window of
// readings is read with one seek.
//
// Both YAML files are flat `key: value` maps; this reader handles that
// subset (comments, blank lines, quoted scalars, document markers) and
// rejects anything else rather than guess.
#include "wfbp_internal.h"

#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>

#define WFBP_API extern "C" __attribute__((visibility("default")))

namespace {

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && isspace((unsigned char)s[a])) a++;
  while (b > a && isspace((unsigned char)s[b - 1])) b--;
  return s.substr(a, b - a);
}

// Flat `key: value` YAML; returns false on a line it cannot read.
bool read_flat_yaml(const char* path, std::map<std::string, std::string>* out) {
  FILE* f = fopen(path, "r");
  if (!f) return false;
  char buf[8192];
  bool ok = true;
  while (fgets(buf, sizeof(buf), f)) {
    std::string line(buf);
    // strip a comment that is not inside quotes
    bool sq = false, dq = false;
    for (size_t i = 0; i < line.size(); i++) {
      if (line[i] == '\'' && !dq) sq = !sq;
      else if (line[i] == '"' && !sq) dq = !dq;
      else if (line[i] == '#' && !sq && !dq && (i == 0 || isspace((unsigned char)line[i - 1]))) {
        line.resize(i);
        break;
      }
    }
    line = trim(line);
    if (line.empty() || line == "---" || line == "...") continue;
    const size_t c = line.find(':');
    if (c == std::string::npos || c == 0) {
      ok = false;
      break;
    }
    std::string key = trim(line.substr(0, c)), val = trim(line.substr(c + 1));
    if (val.size() >= 2 && ((val.front() == '"' && val.back() == '"') || (val.front() == '\'' && val.back() == '\'')))
      val = val.substr(1, val.size() - 2);
    (*out)[key] = val;
  }
  fclose(f);
  return ok;
}

bool to_double(const std::map<std::string, std::string>& m, const char* key, double* v) {
  auto it = m.find(key);
  if (it == m.end()) return false;
  errno = 0;
  char* end = nullptr;
  const double d = strtod(it->second.c_str(), &end);
  if (errno || end == it->second.c_str() || *end) return false;
  *v = d;
  return true;
}

int ffs_mode_from_name(std::string s) {
  for (auto& ch : s) ch = (char)toupper((unsigned char)ch);
  // DICOM-CT-PD mode names (FFSNONE, FFSZ, FFSXY, FFSXYZ) and plain forms
  if (s.empty() || s == "FFSNONE" || s == "NONE") return WFBP_FFS_NONE;
  if (s == "FFSZ" || s == "Z") return WFBP_FFS_Z;
  if (s == "FFSXY" || s == "FFSPHI" || s == "PHI") return WFBP_FFS_PHI;
  if (s == "FFSXYZ" || s == "FFSPHIZ" || s == "FFSZPHI" || s == "PHIZ") return WFBP_FFS_PHIZ;
  return -1;
}

const char* ffs_mode_name(int m) {
  switch (m) {
    case WFBP_FFS_Z: return "FFSZ";
    case WFBP_FFS_PHI: return "FFSXY";
    case WFBP_FFS_PHIZ: return "FFSXYZ";
  }
  return "FFSNONE";
}

}  // namespace

WFBP_API int wfbp_parse_recon_config(const char* path, ReconConfig* rp) {
  if (!path || !rp) return WFBP_ERR_INVALID_ARG;
  std::map<std::string, std::string> m;
  if (!read_flat_yaml(path, &m)) return WFBP_ERR_INVALID_ARG;
  memset(rp, 0, sizeof(*rp));
  auto str = [&](const char* key, char* dst, size_t cap) {
    auto it = m.find(key);
    if (it != m.end()) snprintf(dst, cap, "%s", it->second.c_str());
  };
  str("raw_data_dir", rp->raw_data_dir, sizeof(rp->raw_data_dir));
  str("output_dir", rp->output_dir, sizeof(rp->output_dir));
  // parse_config.cpp:44: output file = <config file>_recon.dat
  snprintf(rp->output_file, sizeof(rp->output_file), "%s_recon.dat", path);
  double v;
  // keys that are absent stay 0, as parse_config leaves them
  if (to_double(m, "start_pos", &v)) rp->start_pos = (float)v;
  if (to_double(m, "end_pos", &v)) rp->end_pos = (float)v;
  if (to_double(m, "recon_fov", &v)) rp->recon_fov = (float)v;
  if (to_double(m, "slice_thickness", &v)) rp->slice_thickness = (float)v;
  if (to_double(m, "slice_pitch", &v)) rp->slice_pitch = (float)v;
  if (to_double(m, "nx", &v)) rp->nx = (size_t)v;
  if (to_double(m, "ny", &v)) rp->ny = (size_t)v;
  if (to_double(m, "recon_kernel", &v)) rp->recon_kernel = (int)v;
  if (to_double(m, "x_origin", &v)) rp->x_origin = (float)v;
  if (to_double(m, "y_origin", &v)) rp->y_origin = (float)v;
  if (to_double(m, "tube_angle_offset", &v)) rp->tube_angle_offset = (float)v;
  if (to_double(m, "adaptive_filtration_s", &v)) rp->adaptive_filtration_s = (float)v;
  if (rp->slice_pitch == 0.0f) rp->slice_pitch = rp->slice_thickness;  // parse_config.cpp:59-60
  return WFBP_OK;
}

WFBP_API int wfbp_read_meta(const char* dir, wfbp_scan_meta* meta) {
  if (!dir || !meta) return WFBP_ERR_INVALID_ARG;
  std::map<std::string, std::string> m;
  const std::string path = std::string(dir) + "/meta.yaml";
  if (!read_flat_yaml(path.c_str(), &m)) return WFBP_ERR_INVALID_ARG;
  memset(meta, 0, sizeof(*meta));
  double v;
  const struct {
    const char* key;
    int kind;  // 0 int, 1 float
    void* dst;
  } fields[] = {
      {"total_num_projections", 0, &meta->total_num_projections},
      {"projections_per_rotation", 0, &meta->projections_per_rotation},
      {"detector_channels", 0, &meta->detector_channels},
      {"detector_rows", 0, &meta->detector_rows},
      {"detector_transverse_spacing", 1, &meta->detector_transverse_spacing},
      {"detector_axial_spacing", 1, &meta->detector_axial_spacing},
      {"detector_central_channel", 1, &meta->detector_central_channel},
      {"detector_central_row", 1, &meta->detector_central_row},
      {"distance_source_to_isocenter", 1, &meta->dist_source_to_isocenter},
      {"distance_source_to_detector", 1, &meta->dist_source_to_detector},
  };
  for (auto& fd : fields) {
    if (!to_double(m, fd.key, &v)) return WFBP_ERR_INVALID_ARG;  // every geometry key is required
    if (fd.kind == 0) *(int*)fd.dst = (int)v;
    else *(float*)fd.dst = (float)v;
  }
  auto it = m.find("flying_focal_spot_mode");
  const int mode = ffs_mode_from_name(it == m.end() ? std::string() : it->second);
  if (mode < 0) return WFBP_ERR_UNSUPPORTED;
  meta->ffs_mode = mode;
  meta->anode_angle = to_double(m, "anode_angle", &v) ? (float)v : 0.0f;
  return WFBP_OK;
}

WFBP_API int wfbp_read_frames(const char* dir, const wfbp_scan_meta* meta, int first, int count, float* tube_angles,
                              float* table_positions, float* raw) {
  if (!dir || !meta || first < 0 || count < 1 || !raw) return WFBP_ERR_INVALID_ARG;
  if (meta->detector_rows < 1 || meta->detector_channels < 1 || first + count > meta->total_num_projections)
    return WFBP_ERR_INVALID_ARG;
  const std::string path = std::string(dir) + "/projections.dat";
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return WFBP_ERR_INVALID_ARG;
  const size_t frame = (size_t)meta->detector_rows * meta->detector_channels;
  const long long stride = (long long)(3 + frame) * (long long)sizeof(float);
  int st = WFBP_OK;
  if (fseeko(f, (off_t)(stride * first), SEEK_SET) != 0) st = WFBP_ERR_INVALID_ARG;
  for (int i = 0; i < count && !st; i++) {
    float hdr[3];
    if (fread(hdr, sizeof(float), 3, f) != 3 || fread(raw + (size_t)i * frame, sizeof(float), frame, f) != frame) {
      st = WFBP_ERR_INVALID_ARG;  // file shorter than the metadata says
      break;
    }
    if (tube_angles) tube_angles[i] = hdr[0];
    if (table_positions) table_positions[i] = hdr[1];
  }
  fclose(f);
  return st;
}

WFBP_API int wfbp_write_scan(const char* dir, const wfbp_scan_meta* meta, const float* tube_angles,
                             const float* table_positions, const float* raw) {
  if (!dir || !meta || !tube_angles || !table_positions || !raw) return WFBP_ERR_INVALID_ARG;
  const std::string mp = std::string(dir) + "/meta.yaml", pp = std::string(dir) + "/projections.dat";
  FILE* f = fopen(mp.c_str(), "w");
  if (!f) return WFBP_ERR_INVALID_ARG;
  fprintf(f, "# FREECT SCAN (written by freect_b200)\n\n# DETECTOR\n");
  fprintf(f, "manufacturer: synthetic\n");
  fprintf(f, "detector_rows: %d\n", meta->detector_rows);
  fprintf(f, "detector_channels: %d\n", meta->detector_channels);
  fprintf(f, "detector_transverse_spacing: %.9g\n", meta->detector_transverse_spacing);
  fprintf(f, "detector_axial_spacing: %.9g\n", meta->detector_axial_spacing);
  fprintf(f, "detector_shape: cylindrical\n\n# SCANNER GEOMETRY\n");
  fprintf(f, "distance_source_to_detector: %.9g\n", meta->dist_source_to_detector);
  fprintf(f, "distance_source_to_isocenter: %.9g\n", meta->dist_source_to_isocenter);
  fprintf(f, "detector_central_row: %.9g\n", meta->detector_central_row);
  fprintf(f, "detector_central_channel: %.9g\n", meta->detector_central_channel);
  fprintf(f, "projection_geometry: fanbeam\n\n# SCAN\n");
  fprintf(f, "scan_type: helical\n");
  fprintf(f, "projections_per_rotation: %d\n", meta->projections_per_rotation);
  fprintf(f, "flying_focal_spot_mode: %s\n", ffs_mode_name(meta->ffs_mode));
  fprintf(f, "total_num_projections: %d\n", meta->total_num_projections);
  const bool ok_meta = fclose(f) == 0;
  if (!ok_meta) return WFBP_ERR_INVALID_ARG;
  f = fopen(pp.c_str(), "wb");
  if (!f) return WFBP_ERR_INVALID_ARG;
  const size_t frame = (size_t)meta->detector_rows * meta->detector_channels;
  bool ok = true;
  for (int i = 0; i < meta->total_num_projections && ok; i++) {
    const float hdr[3] = {tube_angles[i], table_positions[i], meta->dist_source_to_isocenter};
    ok = fwrite(hdr, sizeof(float), 3, f) == 3 && fwrite(raw + (size_t)i * frame, sizeof(float), frame, f) == frame;
  }
  ok = (fclose(f) == 0) && ok;
  return ok ? WFBP_OK : WFBP_ERR_INVALID_ARG;
}
