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

#include <dirent.h>
#include <sys/stat.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

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

// ---------------------------------------------------------------------------
// DICOM-CT-PD projection data (the TCIA LDCT raw-projection format)
// ---------------------------------------------------------------------------
//
// fct_read's DicomDataSet (modules/fct_read/src/DicomDataSet.cpp) reads one
// reading per file through DCMTK: the directory's files sorted by name
// (:156-162), the scan metadata from the first file (readMetadata, :232-316)
// and per file the focal-centre angle / axial position / radial distance,
// the detector size, the rescale slope and intercept, the flying-focal-spot
// shifts and the uint16 pixel data (DicomFrame::readFromFile, :56-155), with
// the private tags of its dictionary (:171-211). DCMTK is not available here,
// so this is a small DICOM Part 10 reader of its own for exactly those
// elements: the file meta group (explicit VR little endian) selects implicit
// or explicit VR little endian for the data set (other transfer syntaxes are
// rejected); top-level elements are scanned, sequences of defined or
// undefined length are skipped.
namespace {

struct DcmElem {
  std::string vr;  // two letters (implicit VR: from the table below)
  const uint8_t* p = nullptr;
  uint32_t len = 0;
};

uint16_t rd16(const uint8_t* p) { return (uint16_t)(p[0] | (p[1] << 8)); }
uint32_t rd32(const uint8_t* p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24); }

// VR of the elements this reader uses, for implicit-VR files (DicomDataSet.cpp:177-210)
const char* implicit_vr(uint32_t tag) {
  switch (tag) {
    case 0x00080070: return "LO";
    case 0x00280010: case 0x00280011: return "US";
    case 0x00281052: case 0x00281053: return "DS";
    case 0x70291010: case 0x70291011: case 0x70331013: return "US";
    case 0x70291002: case 0x70291006: case 0x70311001: case 0x70311002: case 0x70311003: case 0x70311031:
    case 0x70311033: case 0x7033100B: case 0x7033100C: case 0x7033100D: return "FL";
    case 0x7029100B: case 0x7033100E: case 0x70371009: case 0x7037100A: return "CS";
    case 0x7FE00010: return "OW";
    default: return "UN";
  }
}

bool long_form(const std::string& vr) {
  return vr == "OB" || vr == "OW" || vr == "OF" || vr == "OD" || vr == "OL" || vr == "OV" || vr == "SQ" ||
         vr == "UT" || vr == "UN" || vr == "UC" || vr == "UR" || vr == "SV" || vr == "UV";
}

// Skips the items of a sequence of undefined length starting at `i`; returns
// the offset after its delimiter, or 0 on malformed data.
size_t skip_undefined_sequence(const std::vector<uint8_t>& b, size_t i, bool explicit_vr);

// Skips one item (FFFE,E000) of defined or undefined length at `i`.
size_t skip_item(const std::vector<uint8_t>& b, size_t i, bool explicit_vr) {
  if (i + 8 > b.size()) return 0;
  const uint32_t tag = ((uint32_t)rd16(&b[i]) << 16) | rd16(&b[i + 2]);
  const uint32_t len = rd32(&b[i + 4]);
  i += 8;
  if (tag == 0xFFFEE0DDu) return i;  // sequence delimiter (caller handles)
  if (tag != 0xFFFEE000u) return 0;
  if (len != 0xFFFFFFFFu) return i + len <= b.size() ? i + len : 0;
  // undefined-length item: elements until the item delimiter
  while (i + 8 <= b.size()) {
    const uint32_t t = ((uint32_t)rd16(&b[i]) << 16) | rd16(&b[i + 2]);
    if (t == 0xFFFEE00Du) return i + 8;
    std::string vr;
    uint32_t l;
    size_t h;
    if (explicit_vr) {
      vr.assign((const char*)&b[i + 4], 2);
      if (long_form(vr)) { if (i + 12 > b.size()) return 0; l = rd32(&b[i + 8]); h = 12; }
      else { l = rd16(&b[i + 6]); h = 8; }
    } else {
      l = rd32(&b[i + 4]);
      h = 8;
      vr = l == 0xFFFFFFFFu ? "SQ" : "UN";
    }
    i += h;
    if (l == 0xFFFFFFFFu) {
      i = skip_undefined_sequence(b, i, explicit_vr);
      if (!i) return 0;
    } else {
      if (i + l > b.size()) return 0;
      i += l;
    }
  }
  return 0;
}

size_t skip_undefined_sequence(const std::vector<uint8_t>& b, size_t i, bool explicit_vr) {
  while (i + 8 <= b.size()) {
    const uint32_t tag = ((uint32_t)rd16(&b[i]) << 16) | rd16(&b[i + 2]);
    if (tag == 0xFFFEE0DDu) return i + 8;
    i = skip_item(b, i, explicit_vr);
    if (!i) return 0;
  }
  return 0;
}

// Reads a DICOM Part 10 file and collects its top-level elements.
bool dcm_parse(const std::string& path, std::vector<uint8_t>* buf, std::map<uint32_t, DcmElem>* out,
               std::string* err) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) {
    *err = "cannot open " + path;
    return false;
  }
  fseek(f, 0, SEEK_END);
  const long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  buf->resize(n > 0 ? (size_t)n : 0);
  const bool rd_ok = n > 0 && fread(buf->data(), 1, (size_t)n, f) == (size_t)n;
  fclose(f);
  if (!rd_ok) {
    *err = "cannot read " + path;
    return false;
  }
  const std::vector<uint8_t>& b = *buf;
  size_t i = 0;
  if (b.size() >= 132 && memcmp(&b[128], "DICM", 4) == 0) i = 132;
  else if (b.size() >= 4 && memcmp(&b[0], "DICM", 4) == 0) i = 4;
  else {
    *err = path + ": not a DICOM Part 10 file (no DICM marker)";
    return false;
  }
  bool explicit_vr = true;  // the file meta group is always explicit VR little endian
  bool in_meta = true;
  while (i + 8 <= b.size()) {
    const uint16_t grp = rd16(&b[i]), el = rd16(&b[i + 2]);
    const uint32_t tag = ((uint32_t)grp << 16) | el;
    if (in_meta && grp != 0x0002) {
      in_meta = false;
      auto ts = out->find(0x00020010u);
      std::string syntax = ts == out->end() ? "" : std::string((const char*)ts->second.p, ts->second.len);
      while (!syntax.empty() && (syntax.back() == '\0' || syntax.back() == ' ')) syntax.pop_back();
      if (syntax == "1.2.840.10008.1.2") explicit_vr = false;
      else if (syntax == "1.2.840.10008.1.2.1" || syntax.empty()) explicit_vr = true;
      else {
        *err = path + ": unsupported transfer syntax " + syntax + " (implicit or explicit VR little endian only)";
        return false;
      }
    }
    DcmElem e;
    size_t h;
    if (explicit_vr) {
      e.vr.assign((const char*)&b[i + 4], 2);
      if (long_form(e.vr)) {
        if (i + 12 > b.size()) break;
        e.len = rd32(&b[i + 8]);
        h = 12;
      } else {
        e.len = rd16(&b[i + 6]);
        h = 8;
      }
    } else {
      e.vr = implicit_vr(tag);
      e.len = rd32(&b[i + 4]);
      h = 8;
    }
    i += h;
    if (e.len == 0xFFFFFFFFu) {  // a sequence (or encapsulated data) of undefined length
      if (tag == 0x7FE00010u) {
        *err = path + ": encapsulated (compressed) pixel data is not supported";
        return false;
      }
      i = skip_undefined_sequence(b, i, explicit_vr);
      if (!i) {
        *err = path + ": malformed sequence";
        return false;
      }
      continue;
    }
    if (i + e.len > b.size()) {
      *err = path + ": element runs past the end of the file";
      return false;
    }
    e.p = &b[i];
    (*out)[tag] = e;
    i += e.len;
  }
  return true;
}

bool dcm_float(const std::map<uint32_t, DcmElem>& m, uint32_t tag, int index, double* v) {
  auto it = m.find(tag);
  if (it == m.end()) return false;
  const DcmElem& e = it->second;
  if (e.vr == "FL") {
    if (e.len < 4u * (index + 1)) return false;
    float f;
    memcpy(&f, e.p + 4 * index, 4);
    *v = f;
    return true;
  }
  if (e.vr == "FD") {
    if (e.len < 8u * (index + 1)) return false;
    double d;
    memcpy(&d, e.p + 8 * index, 8);
    *v = d;
    return true;
  }
  if (e.vr == "US") {
    if (e.len < 2u * (index + 1)) return false;
    *v = rd16(e.p + 2 * index);
    return true;
  }
  if (e.vr == "DS" || e.vr == "IS") {  // decimal string, values separated by backslashes
    std::string s((const char*)e.p, e.len);
    for (int k = 0; k < index; k++) {
      const size_t bs = s.find('\\');
      if (bs == std::string::npos) return false;
      s = s.substr(bs + 1);
    }
    s = trim(s.substr(0, s.find('\\')));
    while (!s.empty() && s.back() == '\0') s.pop_back();
    errno = 0;
    char* end = nullptr;
    const double d = strtod(s.c_str(), &end);
    if (errno || end == s.c_str()) return false;
    *v = d;
    return true;
  }
  return false;
}

std::string dcm_string(const std::map<uint32_t, DcmElem>& m, uint32_t tag) {
  auto it = m.find(tag);
  if (it == m.end()) return std::string();
  std::string s((const char*)it->second.p, it->second.len);
  while (!s.empty() && (s.back() == '\0' || s.back() == ' ')) s.pop_back();
  return trim(s);
}

// The directory's regular files, sorted by name (DicomDataSet::initialize).
bool dcm_files(const char* dir, std::vector<std::string>* files) {
  DIR* d = opendir(dir);
  if (!d) return false;
  while (dirent* e = readdir(d)) {
    const std::string name = e->d_name;
    if (name == "." || name == "..") continue;
    const std::string path = std::string(dir) + "/" + name;
    struct stat st;
    if (stat(path.c_str(), &st) == 0 && S_ISREG(st.st_mode)) files->push_back(path);
  }
  closedir(d);
  std::sort(files->begin(), files->end());
  return true;
}

}  // namespace

WFBP_API int wfbp_dicom_read_meta(const char* dir, wfbp_scan_meta* meta) {
  if (!dir || !meta) return WFBP_ERR_INVALID_ARG;
  std::vector<std::string> files;
  if (!dcm_files(dir, &files) || files.empty()) return WFBP_ERR_INVALID_ARG;
  std::vector<uint8_t> buf;
  std::map<uint32_t, DcmElem> m;
  std::string err;
  if (!dcm_parse(files[0], &buf, &m, &err)) return WFBP_ERR_INVALID_ARG;
  // DicomDataSet::readMetadata (DicomDataSet.cpp:232-316)
  double rows, chans, dt, da, sid, sdd, ppr, c0, r0;
  if (!dcm_float(m, 0x70291010u, 0, &rows) || !dcm_float(m, 0x70291011u, 0, &chans) ||
      !dcm_float(m, 0x70291002u, 0, &dt) || !dcm_float(m, 0x70291006u, 0, &da) ||
      !dcm_float(m, 0x70311003u, 0, &sid) || !dcm_float(m, 0x70311031u, 0, &sdd) ||
      !dcm_float(m, 0x70331013u, 0, &ppr) || !dcm_float(m, 0x70311033u, 0, &c0) || !dcm_float(m, 0x70311033u, 1, &r0))
    return WFBP_ERR_INVALID_ARG;
  memset(meta, 0, sizeof(*meta));
  meta->total_num_projections = (int)files.size();
  meta->projections_per_rotation = (int)ppr;
  meta->detector_channels = (int)chans;
  meta->detector_rows = (int)rows;
  meta->detector_transverse_spacing = (float)dt;
  meta->detector_axial_spacing = (float)da;
  meta->detector_central_channel = (float)c0;  // (7031,1033)[0]: channel, [1]: row (DicomDataSet.cpp:302-309)
  meta->detector_central_row = (float)r0;
  meta->dist_source_to_isocenter = (float)sid;
  meta->dist_source_to_detector = (float)sdd;
  meta->ffs_mode = ffs_mode_from_name(dcm_string(m, 0x7033100Eu));
  meta->anode_angle = 0.0f;
  return meta->ffs_mode < 0 ? WFBP_ERR_INVALID_ARG : WFBP_OK;
}

WFBP_API int wfbp_dicom_read_frames(const char* dir, const wfbp_scan_meta* meta, int first, int count,
                                    float* tube_angles, float* table_positions, float* raw) {
  if (!dir || !meta || !raw || first < 0 || count < 1) return WFBP_ERR_INVALID_ARG;
  std::vector<std::string> files;
  if (!dcm_files(dir, &files) || (size_t)first + count > files.size()) return WFBP_ERR_INVALID_ARG;
  const int nr = meta->detector_rows, nch = meta->detector_channels;
  const size_t frame = (size_t)nr * nch;
  std::vector<uint8_t> buf;
  for (int k = 0; k < count; k++) {
    std::map<uint32_t, DcmElem> m;
    std::string err;
    buf.clear();
    if (!dcm_parse(files[first + k], &buf, &m, &err)) return WFBP_ERR_INVALID_ARG;
    // DicomFrame::readFromFile (DicomDataSet.cpp:56-155)
    double ang, ax, frows, fch, slope, icpt, irows, icols;
    if (!dcm_float(m, 0x70311001u, 0, &ang) || !dcm_float(m, 0x70311002u, 0, &ax) ||
        !dcm_float(m, 0x70291010u, 0, &frows) || !dcm_float(m, 0x70291011u, 0, &fch) ||
        !dcm_float(m, 0x00281052u, 0, &icpt) || !dcm_float(m, 0x00281053u, 0, &slope) ||
        !dcm_float(m, 0x00280010u, 0, &irows) || !dcm_float(m, 0x00280011u, 0, &icols))
      return WFBP_ERR_INVALID_ARG;
    if ((int)frows != nr || (int)fch != nch) return WFBP_ERR_INVALID_ARG;
    auto px = m.find(0x7FE00010u);
    if (px == m.end() || px->second.len < 2 * frame) return WFBP_ERR_INVALID_ARG;
    const uint8_t* d = px->second.p;
    float* out = raw + (size_t)k * frame;
    const float fs = (float)slope, fi = (float)icpt;
    if ((int)irows == nr && (int)icols == nch) {
      // image rows are detector rows: row-major [rows][channels]
      for (size_t j = 0; j < frame; j++) out[j] = fs * (float)rd16(d + 2 * j) + fi;
    } else if ((int)irows == nch && (int)icols == nr) {
      // image rows are detector channels: the matrix [rows][channels] stored column-major
      for (int r = 0; r < nr; r++)
        for (int c = 0; c < nch; c++) out[(size_t)r * nch + c] = fs * (float)rd16(d + 2 * ((size_t)c * nr + r)) + fi;
    } else {
      return WFBP_ERR_INVALID_ARG;  // Rows/Columns match neither detector orientation
    }
    if (tube_angles) tube_angles[k] = (float)ang;
    if (table_positions) table_positions[k] = (float)ax;
  }
  return WFBP_OK;
}
