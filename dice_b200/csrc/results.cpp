// results.cpp -- DICe text results: the Output_Spec writer and the DICe_Diff
// comparator (host C++).
//
// Writer: the information block, header and rows of Output_Spec::write_info
// / write_header / write_frame (DICe_Schema.cpp:4797-4943) and the file
// naming of Schema::write_output (:4327-4478).  Every value is rounded to
// float before "%4.4E", as the reference prints a scalar_t.
//
// Comparator: DICe_Diff (tools/DICe_Diff.cpp).  Lines are tokenised on ' ',
// ',' and '\r' and upper-cased (tokenize_line); a line of file A whose second
// token contains "DIGITAL" (the masthead) is skipped; numbers compare by
// |(a - b) / a| <= tol in float, skipped when |a| + |b| < 1e-8 or (with a
// floor) |a| < floor; other tokens must be equal unless numerical_only.  The
// parallel form keeps the reference's arithmetic for that path, which
// compares |a - b| for a != 0.
#include <algorithm>
#include <cctype>
#include <cstdarg>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "dicegpu.h"
#include "dicegpu_results.h"

namespace {

// a column of the output: a field-row column, an uncertainty column, a VSG
// column, or 0
struct Column {
  std::string name;
  int src;   // 0: field row, 1: uncertainty row, 2: always 0, 3: VSG row
  int col;
};

bool lookup(const std::string& name, Column& c) {
  static const std::map<std::string, std::pair<int, int>> table = {
      {"COORDINATE_X", {0, DICEGPU_F_COORD_X}},
      {"COORDINATE_Y", {0, DICEGPU_F_COORD_Y}},
      {"DISPLACEMENT_X", {0, DICEGPU_F_DISP_X}},
      {"DISPLACEMENT_Y", {0, DICEGPU_F_DISP_Y}},
      {"ROTATION_Z", {0, DICEGPU_F_ROT_Z}},
      {"NORMAL_STRAIN_X", {0, DICEGPU_F_STRETCH_XX}},
      {"NORMAL_STRAIN_Y", {0, DICEGPU_F_STRETCH_YY}},
      {"SHEAR_STRAIN_XY", {0, DICEGPU_F_SHEAR_XY}},
      {"QUAD_A", {0, DICEGPU_F_QUAD_A + 0}}, {"QUAD_B", {0, DICEGPU_F_QUAD_A + 1}},
      {"QUAD_C", {0, DICEGPU_F_QUAD_A + 2}}, {"QUAD_D", {0, DICEGPU_F_QUAD_A + 3}},
      {"QUAD_E", {0, DICEGPU_F_QUAD_A + 4}}, {"QUAD_F", {0, DICEGPU_F_QUAD_A + 5}},
      {"QUAD_G", {0, DICEGPU_F_QUAD_A + 6}}, {"QUAD_H", {0, DICEGPU_F_QUAD_A + 7}},
      {"QUAD_I", {0, DICEGPU_F_QUAD_A + 8}}, {"QUAD_J", {0, DICEGPU_F_QUAD_A + 9}},
      {"QUAD_K", {0, DICEGPU_F_QUAD_A + 10}}, {"QUAD_L", {0, DICEGPU_F_QUAD_A + 11}},
      {"SIGMA", {0, DICEGPU_F_SIGMA}},
      {"GAMMA", {0, DICEGPU_F_GAMMA}},
      {"BETA", {0, DICEGPU_F_BETA}},
      {"NOISE_LEVEL", {0, DICEGPU_F_NOISE}},
      {"CONTRAST_LEVEL", {0, DICEGPU_F_CONTRAST}},
      {"ACTIVE_PIXELS", {0, DICEGPU_F_ACTIVE_PIXELS}},
      {"STATUS_FLAG", {0, DICEGPU_F_STATUS}},
      {"ITERATIONS", {0, DICEGPU_F_ITERATIONS}},
      {"MATCH", {0, DICEGPU_F_MATCH}},
      {"CONDITION_NUMBER", {0, DICEGPU_F_CONDITION}},
      {"OMEGA", {0, DICEGPU_F_OMEGA}},
      {"FIELD_1", {1, 0}}, {"FIELD_2", {1, 1}}, {"FIELD_3", {1, 2}}, {"FIELD_4", {1, 3}},
      {"FIELD_5", {1, 4}}, {"FIELD_6", {1, 5}}, {"FIELD_7", {1, 6}},
      // defined fields of the reference that this path does not compute
      {"FIELD_8", {2, 0}}, {"FIELD_9", {2, 0}}, {"FIELD_10", {2, 0}}, {"SSSIG", {2, 0}},
      {"NEIGHBOR_ID", {2, 0}}, {"DIST_CORRECTED_SUBSET_DISP_X", {2, 0}},
      {"DIST_CORRECTED_SUBSET_DISP_Y", {2, 0}}, {"STEREO_DISPLACEMENT_X", {2, 0}},
      {"STEREO_DISPLACEMENT_Y", {2, 0}}, {"MODEL_DISPLACEMENT_X", {2, 0}}, {"MODEL_DISPLACEMENT_Y", {2, 0}},
      {"MODEL_DISPLACEMENT_Z", {2, 0}}, {"CROSS_EPI_ERROR", {2, 0}}, {"EPI_A", {2, 0}}, {"EPI_B", {2, 0}},
      {"EPI_C", {2, 0}},
      // VSG_Strain_Post_Processor fields (DICe_PostProcessor.h:105-117)
      {"VSG_STRAIN_XX", {3, DICEGPU_VSG_STRAIN_XX}}, {"VSG_STRAIN_YY", {3, DICEGPU_VSG_STRAIN_YY}},
      {"VSG_STRAIN_XY", {3, DICEGPU_VSG_STRAIN_XY}}, {"VSG_DUDX", {3, DICEGPU_VSG_DUDX}},
      {"VSG_DUDY", {3, DICEGPU_VSG_DUDY}}, {"VSG_DVDX", {3, DICEGPU_VSG_DVDX}}, {"VSG_DVDY", {3, DICEGPU_VSG_DVDY}},
  };
  const auto it = table.find(name);
  if (it == table.end()) return false;
  c.name = name;
  c.src = it->second.first;
  c.col = it->second.second;
  return true;
}

const char* interp_name(int m) {
  return m == DICEGPU_BILINEAR ? "BILINEAR" : m == DICEGPU_BICUBIC ? "BICUBIC" : "KEYS_FOURTH";
}
const char* grad_name(int m) { return m == DICEGPU_CONVOLUTION_5_POINT ? "CONVOLUTION_5_POINT" : "FINITE_DIFFERENCE"; }
const char* opt_name(int m) {
  switch (m) {
    case DICEGPU_SIMPLEX: return "SIMPLEX";
    case DICEGPU_GRADIENT_BASED: return "GRADIENT_BASED";
    case DICEGPU_SIMPLEX_THEN_GRADIENT_BASED: return "SIMPLEX_THEN_GRADIENT_BASED";
    default: return "GRADIENT_BASED_THEN_SIMPLEX";
  }
}

void appendf(std::string& s, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
void appendf(std::string& s, const char* fmt, ...) {
  char buf[4096];
  va_list ap;
  va_start(ap, fmt);
  const int n = std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (n > 0) s.append(buf, std::min<size_t>((size_t)n, sizeof(buf) - 1));
}

int give(const std::string& s, char* buf, size_t cap, size_t* len) {
  if (len) *len = s.size();
  if (buf && cap) {
    const size_t k = std::min(cap - 1, s.size());
    std::memcpy(buf, s.data(), k);
    buf[k] = 0;
  }
  return DICEGPU_OK;
}

}  // namespace

struct dicegpu_output {
  dicegpu_params p;
  std::vector<Column> cols;
  std::string delim;
  bool omit_row_id;
  std::string ref_image, def_image, version, init_method;
  int subset_size, step_x, step_y, strain_window, incremental, sort_rows;

  std::string info_text() const {
    std::string s;
    appendf(s, "***\n");
    appendf(s, "*** Digital Image Correlation Engine (DICe) results written by dicegpu (version: %s)\n",
            version.c_str());
    appendf(s, "***\n");
    appendf(s, "*** Reference image: %s \n", ref_image.c_str());
    appendf(s, "*** Deformed image: %s \n", def_image.c_str());
    appendf(s, "*** DIC method : local \n");
    appendf(s, "*** Correlation method: ZNSSD\n");
    appendf(s, "*** Interpolation method: %s\n", interp_name(p.interpolation));
    appendf(s, "*** Image gradient method: %s\n", grad_name(p.gradient_method));
    appendf(s, "*** Optimization method: %s\n", opt_name(p.optimization));
    appendf(s, "*** Projection method: DISPLACEMENT_BASED\n");
    appendf(s, "*** Guess initialization method: %s\n", init_method.c_str());
    appendf(s, "*** Seed location: N/A\n");
    appendf(s, "*** Shape functions: ");
    if (p.shape_function == DICEGPU_QUADRATIC_SF) {
      appendf(s, "quadratic (A,B,C,D,E,F,G,H,I,J,K,L)");
    } else {
      if (p.enable_translation) appendf(s, "Translation (u,v) ");
      if (p.enable_rotation) appendf(s, "Rotation (theta) ");
      if (p.enable_normal_strain) appendf(s, "Normal Strain (ex,ey) ");
      if (p.enable_shear_strain) appendf(s, "Shear Strain (gamma_xy) ");
    }
    appendf(s, "\n");
    appendf(s, "*** Incremental correlation: %s\n", incremental ? "true" : "false");
    appendf(s, "*** Subset size: %i\n", subset_size);
    appendf(s, "*** Step size: x %i y %i (-1 implies not regular grid)\n", step_x, step_y);
    if (strain_window == -1) appendf(s, "*** Strain window: N/A\n");
    else appendf(s, "*** Strain window size in pixels: %i (only first strain post-processor is reported)\n", strain_window);
    appendf(s, "*** Coordinates given with (0,0) as upper left corner of image, x positive right, y positive down\n");
    appendf(s, "***\n");
    return s;
  }
  std::string header_text(const char* row_id) const {
    std::string s;
    if (!omit_row_id) appendf(s, "%s%s", row_id, delim.c_str());
    for (size_t i = 0; i < cols.size(); ++i) appendf(s, "%s%s", i ? delim.c_str() : "", cols[i].name.c_str());
    appendf(s, "\n");
    return s;
  }
  std::string row_text(int row, const double* f, const double* u, const double* g) const {
    std::string s;
    if (!omit_row_id) appendf(s, "%i%s", row, delim.c_str());
    for (size_t i = 0; i < cols.size(); ++i) {
      double v = 0.0;
      if (cols[i].src == 0) v = f[cols[i].col];
      else if (cols[i].src == 1 && u) v = u[cols[i].col];
      else if (cols[i].src == 3 && g) v = g[cols[i].col];
      const float sv = (float)v;
      appendf(s, "%s%4.4E", i ? delim.c_str() : "", (double)sv);
    }
    appendf(s, "\n");
    return s;
  }
};

extern "C" int dicegpu_output_create(const dicegpu_params* params, const char* fields, const char* delimiter,
                                     int omit_row_id, const dicegpu_output_info* info, dicegpu_output** out) {
  if (!params || !out) return DICEGPU_ERR_ARG;
  *out = nullptr;
  dicegpu_output* o = new (std::nothrow) dicegpu_output();
  if (!o) return DICEGPU_ERR_NOMEM;
  o->p = *params;
  o->delim = delimiter ? delimiter : " ";
  o->omit_row_id = omit_row_id != 0;
  o->ref_image = info && info->ref_image ? info->ref_image : "";
  o->def_image = info && info->def_image ? info->def_image : "";
  o->version = info && info->version ? info->version : dicegpu_version();
  o->subset_size = info ? info->subset_size : params->subset_size;
  o->step_x = info ? info->step_size_x : -1;
  o->step_y = info ? info->step_size_y : -1;
  o->strain_window = info ? info->strain_window : -1;
  o->incremental = (info && info->incremental) || params->use_incremental_formulation;
  o->sort_rows = info ? info->sort_rows : 0;
  o->init_method = info && info->initialization_method ? info->initialization_method : "USE_FIELD_VALUES";
  std::vector<std::string> names;
  if (!fields) {
    // Output_Spec's default columns (DICe_Schema.cpp:4683-4696)
    names = {"COORDINATE_X", "COORDINATE_Y", "DISPLACEMENT_X", "DISPLACEMENT_Y", "ROTATION_Z"};
    if (params->shape_function == DICEGPU_AFFINE_SF) {
      names.push_back("NORMAL_STRAIN_X");
      names.push_back("NORMAL_STRAIN_Y");
      names.push_back("SHEAR_STRAIN_XY");
    }
    names.push_back("SIGMA");
    names.push_back("STATUS_FLAG");
  } else {
    std::string cur;
    for (const char* q = fields;; ++q) {
      if (*q == 0 || *q == ',' || *q == ' ' || *q == '\t' || *q == '\n') {
        if (!cur.empty()) names.push_back(cur);
        cur.clear();
        if (*q == 0) break;
      } else {
        cur += (char)std::toupper((unsigned char)*q);
      }
    }
  }
  std::set<std::string> seen;
  for (const auto& n : names) {
    Column c;
    if (!lookup(n, c) || !seen.insert(n).second) {
      delete o;
      return DICEGPU_ERR_ARG;
    }
    o->cols.push_back(c);
  }
  if (o->cols.empty()) {
    delete o;
    return DICEGPU_ERR_ARG;
  }
  *out = o;
  return DICEGPU_OK;
}

extern "C" int dicegpu_output_destroy(dicegpu_output* o) {
  delete o;
  return DICEGPU_OK;
}

extern "C" int dicegpu_output_set_images(dicegpu_output* o, const char* ref_image, const char* def_image) {
  if (!o) return DICEGPU_ERR_ARG;
  if (ref_image) o->ref_image = ref_image;
  if (def_image) o->def_image = def_image;
  return DICEGPU_OK;
}

extern "C" int dicegpu_output_num_fields(const dicegpu_output* o, int* n) {
  if (!o || !n) return DICEGPU_ERR_ARG;
  *n = (int)o->cols.size();
  return DICEGPU_OK;
}

extern "C" int dicegpu_output_info_text(const dicegpu_output* o, char* buf, size_t cap, size_t* len) {
  if (!o) return DICEGPU_ERR_ARG;
  return give(o->info_text(), buf, cap, len);
}

extern "C" int dicegpu_output_header_text(const dicegpu_output* o, const char* row_id, char* buf, size_t cap,
                                          size_t* len) {
  if (!o || !row_id) return DICEGPU_ERR_ARG;
  return give(o->header_text(row_id), buf, cap, len);
}

extern "C" int dicegpu_output_row_text(const dicegpu_output* o, int row_index, const double* fields,
                                       const double* unc, const double* vsg, char* buf, size_t cap, size_t* len) {
  if (!o || !fields) return DICEGPU_ERR_ARG;
  return give(o->row_text(row_index, fields, unc, vsg), buf, cap, len);
}

namespace {
int digits(int v) {
  int d = 0;
  while (v) { v /= 10; ++d; }
  return d;
}
bool write_all(const std::string& path, const std::string& text, const char* mode) {
  std::FILE* f = std::fopen(path.c_str(), mode);
  if (!f) return false;
  const bool ok = std::fwrite(text.data(), 1, text.size(), f) == text.size();
  return std::fclose(f) == 0 && ok;
}
}  // namespace

extern "C" int dicegpu_output_write_frame(const dicegpu_output* o, const char* folder, const char* prefix,
                                          int frame, int first_frame, int num_frames, int n, const double* fields,
                                          const double* unc, const double* vsg, int separate_files) {
  if (!o || !folder || !prefix || !fields || n < 1) return DICEGPU_ERR_ARG;
  const std::string base = std::string(folder) + prefix + "_";
  auto U = [&](int i) { return unc ? unc + (size_t)i * DICEGPU_UNCERTAINTY_STRIDE : nullptr; };
  auto G = [&](int i) { return vsg ? vsg + (size_t)i * DICEGPU_VSG_STRIDE : nullptr; };
  if (separate_files) {
    const int total = digits(n);
    for (int i = 0; i < n; ++i) {
      const int mine = i == 0 ? 1 : digits(i);
      std::string name = base + std::string((size_t)std::max(total - mine, 0), '0') + std::to_string(i) + ".txt";
      if (frame == first_frame && !write_all(name, o->info_text() + o->header_text("FRAME"), "w"))
        return DICEGPU_ERR_ARG;
      if (!write_all(name, o->row_text(frame, fields + (size_t)i * DICEGPU_FIELD_STRIDE, U(i), G(i)), "a"))
        return DICEGPU_ERR_ARG;
    }
    return DICEGPU_OK;
  }
  int zeros = 0;
  if (num_frames > 0) {
    const int total = digits(first_frame + num_frames);
    const int mine = frame == 0 ? 1 : digits(frame);
    zeros = std::max(total - mine, 0);
  }
  std::string text = o->info_text() + o->header_text("SUBSET_ID");
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  if (o->sort_rows) {
    // sort_txt_output: by x, then y (DICe_Schema.cpp:4430-4450), on float coordinates
    auto X = [&](int i) { return (float)fields[(size_t)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_COORD_X]; };
    auto Y = [&](int i) { return (float)fields[(size_t)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_COORD_Y]; };
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return X(a) < X(b) || (X(a) == X(b) && Y(a) < Y(b)); });
  }
  for (int i : order) text += o->row_text(i, fields + (size_t)i * DICEGPU_FIELD_STRIDE, U(i), G(i));
  const std::string name = base + std::string((size_t)zeros, '0') + std::to_string(frame) + ".txt";
  return write_all(name, text, "w") ? DICEGPU_OK : DICEGPU_ERR_ARG;
}

// ---------------------------------------------------------------------------
// DICe_Diff
// ---------------------------------------------------------------------------
namespace {

bool get_line(std::istream& is, std::string& t) {
  t.clear();
  if (!is.good()) return false;
  std::streambuf* sb = is.rdbuf();
  bool any = false;
  for (;;) {
    const int c = sb->sbumpc();
    if (c == std::streambuf::traits_type::eof()) {
      is.setstate(std::ios::eofbit);
      return any || !t.empty();
    }
    any = true;
    if (c == '\n') return true;
    if (c == '\r') {
      if (sb->sgetc() == '\n') sb->sbumpc();
      return true;
    }
    t += (char)c;
  }
}

// tokenize_line(file, " ,\r") with capitalisation
std::vector<std::string> tokens(std::istream& is) {
  std::string line;
  get_line(is, line);
  std::vector<std::string> tok;
  std::size_t i = 0;
  auto delim = [](char ch) { return ch == ' ' || ch == ',' || ch == '\r'; };
  while (tok.size() < 100) {
    while (i < line.size() && delim(line[i])) ++i;
    if (i >= line.size()) break;
    std::size_t j = i;
    while (j < line.size() && !delim(line[j])) ++j;
    std::string t = line.substr(i, j - i);
    for (auto& ch : t) ch = (char)std::toupper((unsigned char)ch);
    tok.push_back(t);
    i = j;
  }
  if (!tok.empty() && tok[0].find('#') == 0) tok.clear();
  return tok;
}

bool is_number(const std::string& s) {
  if (s.empty()) return false;
  for (char ch : s)
    if (!(std::isdigit((unsigned char)ch) || ch == '+' || ch == '-' || ch == 'e' || ch == 'E' || ch == '.'))
      return false;
  return true;
}

void report_line(std::string& r, int line, const std::vector<std::string>& a, const std::vector<std::string>& b,
                 const std::vector<std::pair<int, char>>& bad) {
  std::string ids;
  for (const auto& x : bad) ids += std::to_string(x.first) + "[" + x.second + "] ";
  r += "< " + std::to_string(line) + " (" + ids + "): ";
  for (const auto& t : a) r += t + " ";
  r += "\n> " + std::to_string(line) + " (" + ids + "): ";
  for (const auto& t : b) r += t + " ";
  r += "\n";
}

// one line pair; `parallel` selects that path's arithmetic
bool compare_tokens(const std::vector<std::string>& ta, const std::vector<std::string>& tb, float tol, float floor,
                    bool use_floor, bool numerical_only, bool parallel, std::vector<std::pair<int, char>>& bad) {
  bool diff_line = false;
  for (size_t i = 0; i < ta.size(); ++i) {
    if (is_number(ta[i])) {
      const float a = (float)std::strtod(ta[i].c_str(), nullptr);
      const float b = (float)std::strtod(tb[i].c_str(), nullptr);
      float diff;
      bool below;
      if (parallel) {
        diff = a == 0.0f ? std::fabs((a - b) / a) : std::fabs(a - b);
        below = std::fabs(a) < floor && a != 0.0f;
      } else {
        diff = std::fabs((a - b) / a);
        below = std::fabs(a) < floor;
      }
      const bool tiny = std::fabs(a) + std::fabs(b) < 1.0e-8f;
      if (!below || !use_floor) {
        if (!tiny && diff > tol) {
          diff_line = true;
          bad.emplace_back((int)i, 'n');
        }
      }
    } else {
      if (ta[i] != tb[i] && !numerical_only) diff_line = true;
      bad.emplace_back((int)i, 's');
    }
  }
  return diff_line;
}

int diff_serial(std::istream& A, std::istream& B, float tol, float floor, bool use_floor, bool numerical_only,
                std::string& rep) {
  int errors = 0, line = 0;
  while (!A.eof()) {
    if (B.eof()) {
      rep += "Error, File A has more lines than FileB\n";
      ++errors;
      break;
    }
    const auto ta = tokens(A);
    const auto tb = tokens(B);
    if (ta.size() >= 2 && ta[1].find("DIGITAL") != std::string::npos) {
      ++line;
      continue;
    }
    if (ta.size() != tb.size()) {
      rep += "Error, Different number of tokens per line A:" + std::to_string(ta.size()) +
             " B: " + std::to_string(tb.size()) + "\n";
      ++errors;
      break;
    }
    std::vector<std::pair<int, char>> bad;
    if (compare_tokens(ta, tb, tol, floor, use_floor, numerical_only, false, bad)) {
      ++errors;
      report_line(rep, line, ta, tb, bad);
    }
    ++line;
  }
  return errors;
}

}  // namespace

extern "C" int dicegpu_diff_text(const char* a, size_t a_len, const char* b, size_t b_len, double rel_tol,
                                 double floor, int use_floor, int numerical_only, int* failed, char* report,
                                 size_t cap) {
  if (!a || !b || !failed) return DICEGPU_ERR_ARG;
  std::istringstream A(std::string(a, a_len)), B(std::string(b, b_len));
  std::string rep;
  *failed = diff_serial(A, B, (float)rel_tol, (float)floor, use_floor != 0, numerical_only != 0, rep);
  give(rep, report, cap, nullptr);
  return DICEGPU_OK;
}

extern "C" int dicegpu_diff_files(const char* a, const char* b, double rel_tol, double floor, int use_floor,
                                  int numerical_only, int num_procs, int* failed, char* report, size_t cap) {
  if (!a || !b || !failed) return DICEGPU_ERR_ARG;
  std::ifstream A(a, std::ios::in | std::ios::binary);
  if (!A.good()) return DICEGPU_ERR_ARG;
  const float tol = (float)rel_tol, fl = (float)floor;
  std::string rep;
  int errors = 0;
  if (num_procs <= 1) {
    std::ifstream B(b, std::ios::in | std::ios::binary);
    if (!B.good()) return DICEGPU_ERR_ARG;
    errors = diff_serial(A, B, tol, fl, use_floor != 0, numerical_only != 0, rep);
  } else {
    // rows of A by their leading id; pieces <b>.<procs>.<i>.txt compared by id
    std::map<int, std::vector<std::string>> rows;
    while (!A.eof()) {
      const auto t = tokens(A);
      if (t.empty() || !is_number(t[0])) continue;
      const double id = std::strtod(t[0].c_str(), nullptr);
      if (id != std::floor(id)) return DICEGPU_ERR_ARG;   // the first column must be an id
      rows.insert(std::make_pair((int)std::strtol(t[0].c_str(), nullptr, 0), t));
    }
    std::set<int> seen;
    for (int p = 0; p < num_procs; ++p) {
      const std::string name = std::string(b) + "." + std::to_string(num_procs) + "." + std::to_string(p) + ".txt";
      std::ifstream B(name, std::ios::in | std::ios::binary);
      if (!B.good()) return DICEGPU_ERR_ARG;
      int line = 0;
      while (!B.eof()) {
        const auto tb = tokens(B);
        if (tb.empty() || !is_number(tb[0])) continue;
        const int id = (int)std::strtol(tb[0].c_str(), nullptr, 0);
        const auto it = rows.find(id);
        if (it == rows.end()) return DICEGPU_ERR_ARG;
        seen.insert(id);
        const auto& ta = it->second;
        if (ta.size() != tb.size()) {
          rep += "Error, output files are not compatible (read error)\n";
          ++errors;
          break;
        }
        std::vector<std::pair<int, char>> bad;
        if (compare_tokens(ta, tb, tol, fl, use_floor != 0, numerical_only != 0, true, bad)) {
          ++errors;
          report_line(rep, line, ta, tb, bad);
        }
        ++line;
      }
    }
    for (const auto& kv : rows)
      if (!seen.count(kv.first)) {
        rep += "Error, some ids in the serial output file were not present in any of the parallel output files\n";
        ++errors;
        break;
      }
  }
  *failed = errors;
  give(rep, report, cap, nullptr);
  return DICEGPU_OK;
}
