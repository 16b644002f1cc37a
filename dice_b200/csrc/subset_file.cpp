// subset_file.cpp -- DICe subset files: parser and hand-off to a context.
//
// The grammar, the token rules and the checks follow read_subset_file and
// read_shapes (DICe_Parser.cpp:1098-1860): lines are split on blanks and
// tabs and upper-cased; a line whose first token starts with '#' is a
// comment; integers are read with strtol base 0 and reals with strtod, after
// is_number accepted the token.  Parsed content lands in plain arrays that
// map one to one onto the C ABI (dicegpu_shape rows, CSR blocking lists).
#include <algorithm>
#include <cctype>
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
#include "dicegpu_subset_file.h"

namespace {

struct Seed {
  double v[6] = {0, 0, 0, 0, 0, 0};   // u, v, ex, ey, gxy, theta
  int flags = 0;
  int loc_x = 0, loc_y = 0;           // LOCATION (region-of-interest seeds)
};

struct ShapeDef {
  dicegpu_shape s;
  std::vector<int32_t> vx, vy;
};

struct ConformalDef {
  std::vector<ShapeDef> shapes;   // roles set
};

}  // namespace

struct dicegpu_subset_file {
  std::vector<double> coords;                    // x, y pairs
  bool roi = false;
  std::map<int, ConformalDef> conformal;         // first definition of an id wins
  std::map<int, std::vector<int>> blocking;
  std::set<int> force_simplex;
  std::map<int, Seed> seeds;
  std::map<int, int> features;
  std::map<int, std::vector<int32_t>> skip_solve;   // SKIP_SOLVE frame ids, ascending
  int n_roi = 0;
};

namespace {

struct ParseError {
  std::string msg;
};

[[noreturn]] void fail(const std::string& m) { throw ParseError{m}; }

// safeGetline (DICe_Parser.cpp:1007-1042): \n, \r\n and \r all end a line.
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

const std::size_t kMaxTokens = 100;   // MAX_TOKENS_PER_LINE

// tokenize_line (DICe_Parser.cpp:1044-1085)
std::vector<std::string> tokenize(std::istream& is, bool* got_line = nullptr, bool upper = true) {
  std::string line;
  const bool ok = get_line(is, line);
  if (got_line) *got_line = ok;
  std::vector<std::string> tok;
  std::size_t i = 0;
  while (tok.size() < kMaxTokens) {
    while (i < line.size() && (line[i] == ' ' || line[i] == '\t')) ++i;
    if (i >= line.size()) break;
    std::size_t j = i;
    while (j < line.size() && line[j] != ' ' && line[j] != '\t') ++j;
    std::string t = line.substr(i, j - i);
    if (upper)
      for (auto& ch : t) ch = (char)std::toupper((unsigned char)ch);
    tok.push_back(t);
    i = j;
  }
  if (!tok.empty() && tok[0].find('#') == 0) tok.clear();   // comment line
  return tok;
}

// is_number (DICe_Parser.cpp:1088-1095)
bool is_number(const std::string& s) {
  if (s.empty()) return false;
  for (char ch : s)
    if (!(std::isdigit((unsigned char)ch) || ch == '+' || ch == '-' || ch == 'e' || ch == 'E' || ch == '.'))
      return false;
  return true;
}
int to_int(const std::string& s) { return (int)std::strtol(s.c_str(), nullptr, 0); }
double to_real(const std::string& s) { return std::strtod(s.c_str(), nullptr); }

bool more(std::istream& is) { return is.good() && !is.eof(); }

// read_circle (DICe_Parser.cpp:1652-1693)
ShapeDef read_circle(std::istream& is) {
  int cx = -1, cy = -1;
  double r = -1.0;
  while (more(is)) {
    const auto t = tokenize(is);
    if (t.empty()) continue;
    if (t[0] == "END") break;
    if (t[0] == "CENTER") {
      if (t.size() < 3) fail("not enough values to define circle center point");
      if (!is_number(t[1]) || !is_number(t[2])) fail("circle center: both tokens should be numbers");
      cx = to_int(t[1]);
      cy = to_int(t[2]);
    } else if (t[0] == "RADIUS") {
      if (t.size() < 2) fail("not enough values to define circle radius");
      if (!is_number(t[1])) fail("circle radius should be a number");
      r = to_real(t[1]);
    } else {
      fail("invalid token in circle definition " + t[0]);
    }
  }
  if (r == -1.0 || cx == -1 || cy == -1) fail("incomplete circle definition");
  ShapeDef d;
  std::memset(&d.s, 0, sizeof(d.s));
  d.s.kind = DICEGPU_SHAPE_CIRCLE;
  d.s.cx = cx;
  d.s.cy = cy;
  d.s.radius = (float)r;
  return d;
}

// read_rectangle (DICe_Parser.cpp:1695-1790)
ShapeDef read_rectangle(std::istream& is) {
  int cx = -1, cy = -1, width = -1, height = -1;
  int ulx = -1, uly = -1, lrx = -1, lry = -1;
  bool corners = false;
  while (more(is)) {
    const auto t = tokenize(is);
    if (t.empty()) continue;
    if (t[0] == "END") break;
    if (t[0] == "CENTER") {
      if (t.size() < 3) fail("not enough values to define rectangle center point");
      if (!is_number(t[1]) || !is_number(t[2])) fail("rectangle center: both tokens should be numbers");
      cx = to_int(t[1]);
      cy = to_int(t[2]);
    } else if (t[0] == "WIDTH" || t[0] == "HEIGHT") {
      if (t.size() < 2) fail("not enough values to define the rectangle " + t[0]);
      if (!is_number(t[1])) fail("rectangle " + t[0] + " should be a number");
      (t[0] == "WIDTH" ? width : height) = (int)to_real(t[1]);
    } else if (t[0] == "UPPER_LEFT" || t[0] == "LOWER_RIGHT") {
      if (t.size() < 3) fail("not enough values to define rectangle " + t[0]);
      if (!is_number(t[1]) || !is_number(t[2])) fail("rectangle " + t[0] + ": both tokens should be numbers");
      corners = true;
      if (t[0] == "UPPER_LEFT") { ulx = to_int(t[1]); uly = to_int(t[2]); }
      else { lrx = to_int(t[1]); lry = to_int(t[2]); }
    } else {
      fail("invalid token in rectangle definition " + t[0]);
    }
  }
  if (corners) {
    if (ulx < 0 || uly < 0 || lrx < 0 || lry < 0) fail("rectangle corner missing or negative");
    if (lrx < ulx) fail("rectangle inverted or zero width");
    if (lry < uly) fail("rectangle inverted or zero height");
    width = lrx - ulx;
    height = lry - uly;
    cx = width / 2 + ulx;
    cy = height / 2 + uly;
  }
  if (width <= 0 || height <= 0 || cx < 0 || cy < 0) fail("invalid rectangle");
  ShapeDef d;
  std::memset(&d.s, 0, sizeof(d.s));
  d.s.kind = DICEGPU_SHAPE_RECTANGLE;
  d.s.cx = cx;
  d.s.cy = cy;
  d.s.width = width;
  d.s.height = height;
  return d;
}

// read_polygon (DICe_Parser.cpp:1792-1832)
ShapeDef read_polygon(std::istream& is) {
  ShapeDef d;
  std::memset(&d.s, 0, sizeof(d.s));
  d.s.kind = DICEGPU_SHAPE_POLYGON;
  while (more(is)) {
    const auto t = tokenize(is);
    if (t.empty()) continue;
    if (t[0] == "END") break;
    if (t.size() < 2 || t[0] != "BEGIN" || t[1] != "VERTICES") fail("a polygon holds a BEGIN VERTICES block");
    while (more(is)) {
      const auto v = tokenize(is);
      if (v.empty()) continue;
      if (v[0] == "END") break;
      if (v.size() < 2 || !is_number(v[0]) || !is_number(v[1])) fail("invalid polygon vertex");
      d.vx.push_back(to_int(v[0]));
      d.vy.push_back(to_int(v[1]));
    }
  }
  // the Polygon constructor requires three vertices (DICe_Shape.cpp:53-55)
  if (d.vx.size() < 3) fail("a polygon needs at least three vertices");
  d.s.vertex_count = (int32_t)d.vx.size();
  return d;
}

// read_shapes (DICe_Parser.cpp:1834-1858)
std::vector<ShapeDef> read_shapes(std::istream& is, int role) {
  std::vector<ShapeDef> out;
  while (more(is)) {
    const auto t = tokenize(is);
    if (t.empty()) continue;
    if (t[0] == "END") break;
    if (t.size() < 2 || t[0] != "BEGIN") fail("expected BEGIN <shape>");
    if (t[1] == "CIRCLE") out.push_back(read_circle(is));
    else if (t[1] == "POLYGON") out.push_back(read_polygon(is));
    else if (t[1] == "RECTANGLE") out.push_back(read_rectangle(is));
    else fail("unrecognized shape: " + t[1]);
    out.back().s.role = role;
  }
  if (out.empty()) fail("a shape set needs at least one shape");
  return out;
}

// a SEED block (conformal: no LOCATION; region of interest: LOCATION required)
Seed read_seed(std::istream& is, bool roi) {
  Seed sd;
  bool has_loc = false;
  while (more(is)) {
    const auto t = tokenize(is);
    if (t.empty()) continue;
    if (t[0] == "END") break;
    if (t[0] == "LOCATION") {
      if (!roi) fail("a conformal subset's seed takes no location (the centroid is used)");
      if (t.size() <= 2 || !is_number(t[1]) || !is_number(t[2])) fail("seed location needs x and y");
      has_loc = true;
      sd.loc_x = to_int(t[1]);
      sd.loc_y = to_int(t[2]);
    } else if (t[0] == "DISPLACEMENT" || t[0] == "NORMAL_STRAIN") {
      if (t.size() <= 2 || !is_number(t[1]) || !is_number(t[2])) fail("seed " + t[0] + " needs x and y values");
      const int k = t[0] == "DISPLACEMENT" ? 0 : 2;
      sd.v[k] = to_real(t[1]);
      sd.v[k + 1] = to_real(t[2]);
      sd.flags |= t[0] == "DISPLACEMENT" ? DICEGPU_SF_SEED_DISPLACEMENT : DICEGPU_SF_SEED_NORMAL_STRAIN;
    } else if (t[0] == "SHEAR_STRAIN" || t[0] == "ROTATION") {
      if (t.size() <= 1 || !is_number(t[1])) fail("seed " + t[0] + " needs a value");
      const bool shear = t[0] == "SHEAR_STRAIN";
      sd.v[shear ? 4 : 5] = to_real(t[1]);
      sd.flags |= shear ? DICEGPU_SF_SEED_SHEAR_STRAIN : DICEGPU_SF_SEED_ROTATION;
    } else {
      fail("unrecognized command in seed block " + t[0]);
    }
  }
  if (roi && !has_loc) fail("seed must have location specified");
  if (!(sd.flags & DICEGPU_SF_SEED_DISPLACEMENT)) fail("seed must have at least a displacement guess");
  return sd;
}

void read_coordinates(std::istream& is, dicegpu_subset_file& F) {
  while (more(is)) {
    const auto t = tokenize(is);
    if (t.empty()) continue;
    if (t[0] == "END") break;
    if (!is_number(t[0])) fail("error parsing subset coordinates: " + t[0]);
    if (t.size() < 2 || t[1] == "#") fail("invalid coordinate (not enough values)");
    F.coords.push_back(to_real(t[0]));
    F.coords.push_back(to_real(t[1]));
  }
  if (F.coords.size() < 2) fail("no subset coordinates");
}

// BEGIN REGION_OF_INTEREST (DICe_Parser.cpp:1180-1365): the region's shapes
// and seed are read and checked; boundary conditions only for their form
void read_roi(std::istream& is, dicegpu_subset_file& F) {
  F.roi = true;
  ConformalDef def;
  while (more(is)) {
    const auto t = tokenize(is);
    if (t.empty()) continue;
    if (t[0] == "END") break;
    if (t[0] == "USE_REGULAR_GRID" || t[0] == "ENFORCE_LAGRANGE_BC") continue;
    if (t[0] == "IC_VALUE_X" || t[0] == "IC_VALUE_Y") {
      if (t.size() <= 1 || !is_number(t[1])) fail(t[0] + " needs a value");
    } else if (t[0] == "DIRICHLET_BC") {
      if (t.size() < 7) fail("not enough values specified for dirichlet bc");
      if (!is_number(t[2]) || !is_number(t[3]) || !is_number(t[4]) || !is_number(t[5])) fail("invalid dirichlet bc");
      if (!is_number(t[6]) && !(t[6] == "USE_SUBSETS" && t.size() > 7)) fail("invalid dirichlet bc value");
    } else if (t[0] == "NEUMANN_BC") {
      if (t.size() < 5) fail("not enough values specified for Neumann bc");
      if (!is_number(t[2]) || !is_number(t[3]) || !is_number(t[4])) fail("invalid neumann bc");
    } else if (t[0] == "BEGIN") {
      if (t.size() < 2) fail("BEGIN needs a block name");
      if (t[1] == "BOUNDARY" || t[1] == "EXCLUDED") {
        auto sh = read_shapes(is, t[1] == "BOUNDARY" ? DICEGPU_ROLE_BOUNDARY : DICEGPU_ROLE_EXCLUDED);
        def.shapes.insert(def.shapes.end(), sh.begin(), sh.end());
      } else if (t[1] == "SEED") {
        F.seeds.insert(std::make_pair(F.n_roi, read_seed(is, true)));
      } else {
        fail("error parsing region of interest block " + t[1]);
      }
    } else {
      fail("unknown region of interest command: " + t[0]);
    }
  }
  F.conformal.insert(std::make_pair(F.n_roi, def));
  ++F.n_roi;
}

// BEGIN CONFORMAL_SUBSET (DICe_Parser.cpp:1366-1600)
void read_conformal(std::istream& is, dicegpu_subset_file& F) {
  int id = -1;
  bool has_seed = false, force = false, test_motion = false, motion_window = false, has_skip = false;
  int features = 0;
  std::vector<int32_t> skip;
  Seed seed;
  ConformalDef def;
  std::vector<int> blocking;
  while (more(is)) {
    const auto t = tokenize(is);
    if (t.empty()) continue;
    if (t[0] == "END") break;
    if (t[0] == "SUBSET_ID") {
      if (t.size() < 2 || !is_number(t[1])) fail("SUBSET_ID needs a number");
      id = to_int(t[1]);
    } else if (t[0] == "TEST_FOR_MOTION") {
      test_motion = true;
      features |= DICEGPU_SF_FEATURE_TEST_MOTION;
    } else if (t[0] == "MOTION_WINDOW") {
      motion_window = true;
      features |= DICEGPU_SF_FEATURE_MOTION_WINDOW;
      if (t.size() == 2) {
        if (!is_number(t[1])) fail("MOTION_WINDOW <subset id> needs a number");
      } else {
        if (t.size() < 5) fail("MOTION_WINDOW requires at least 4 arguments");
        for (int m = 1; m < 5; ++m)
          if (!is_number(t[m])) fail("MOTION_WINDOW parameters should be numbers");
      }
    } else if (t[0] == "SKIP_SOLVE") {
      if (t.size() > 1 && !is_number(t[1])) {
        // the frame ids in a file (DICe_Parser.cpp:1440-1452): not read here
        features |= DICEGPU_SF_FEATURE_SKIP_SOLVE;
      } else {
        // frame ids that turn solving off and on (DICe_Parser.cpp:1454-1463)
        has_skip = true;
        skip.clear();
        for (std::size_t m = 1; m < t.size(); ++m) {
          if (!is_number(t[m])) fail("SKIP_SOLVE ids should be numbers");
          skip.push_back((int32_t)to_int(t[m]));
        }
        std::sort(skip.begin(), skip.end());
      }
    } else if (t[0] == "USE_OPTICAL_FLOW") {
      features |= DICEGPU_SF_FEATURE_OPTICAL_FLOW;
    } else if (t[0] == "FORCE_SIMPLEX") {
      force = true;
    } else if (t[0] == "USE_PATH_FILE") {
      if (t.size() < 2 || is_number(t[1])) fail("USE_PATH_FILE needs a file name");
      features |= DICEGPU_SF_FEATURE_PATH_FILE;
    } else if (t.size() >= 2 && t[1] == "SEED") {
      if (has_seed) fail("only one seed allowed per conformal subset");
      has_seed = true;
      seed = read_seed(is, false);
    } else if (t[0] == "BEGIN") {
      if (t.size() < 2) fail("BEGIN needs a block name");
      if (t[1] == "BOUNDARY" || t[1] == "EXCLUDED" || t[1] == "OBSTRUCTED") {
        const int role = t[1] == "BOUNDARY" ? DICEGPU_ROLE_BOUNDARY
                         : t[1] == "EXCLUDED" ? DICEGPU_ROLE_EXCLUDED : DICEGPU_ROLE_OBSTRUCTED;
        auto sh = read_shapes(is, role);
        def.shapes.insert(def.shapes.end(), sh.begin(), sh.end());
      } else if (t[1] == "BLOCKING_SUBSETS") {
        while (more(is)) {
          const auto b = tokenize(is);
          if (b.empty()) continue;
          if (b[0] == "END") break;
          if (!is_number(b[0])) fail("BLOCKING_SUBSETS lists subset ids");
          blocking.push_back(to_int(b[0]));
        }
      } else {
        fail("error parsing subset file: " + t[1]);
      }
    } else {
      fail("error in parsing conformal subset def, unknown block command: " + t[0]);
    }
  }
  if (id < 0) fail("invalid subset id for conformal subset (SUBSET_ID <id> missing)");
  bool boundary = false;
  for (const auto& s : def.shapes) boundary = boundary || s.s.role == DICEGPU_ROLE_BOUNDARY;
  if (!boundary) fail("a conformal subset needs a boundary");
  if (test_motion && !motion_window) fail("cannot test for motion without defining a motion window");
  F.conformal.insert(std::make_pair(id, def));
  F.blocking.insert(std::make_pair(id, blocking));
  if (force) F.force_simplex.insert(id);
  if (has_seed) F.seeds.insert(std::make_pair(id, seed));
  if (features) F.features[id] |= features;
  if (has_skip) F.skip_solve[id] = skip;
}

void parse(std::istream& is, int width, int height, dicegpu_subset_file& F) {
  bool coords = false, conformal = false;
  while (more(is)) {
    const auto t = tokenize(is);
    if (t.empty()) continue;
    if (t.size() < 2) fail("invalid entry: " + t[0]);
    if (t[0] != "BEGIN") continue;
    if (t[1] == "SUBSET_COORDINATES") {
      coords = true;
      read_coordinates(is, F);
    } else if (t[1] == "REGION_OF_INTEREST") {
      read_roi(is, F);
    } else if (t[1] == "CONFORMAL_SUBSET") {
      conformal = true;
      read_conformal(is, F);
    } else {
      fail("unknown block command: " + t[1]);
    }
  }
  if (F.roi && (coords || conformal))
    fail("with a region of interest, neither coordinates nor conformal subsets can be given");
  for (std::size_t i = 0; i < F.coords.size(); i += 2) {
    const double x = F.coords[i], y = F.coords[i + 1];
    if (x < 0 || (x >= width && width != -1)) fail("invalid subset coordinate x: " + std::to_string(x));
    if (y < 0 || (y >= height && height != -1)) fail("invalid subset coordinate y: " + std::to_string(y));
  }
}

int finish(std::istream& is, int width, int height, dicegpu_subset_file** out, char* err, int err_len) {
  dicegpu_subset_file* F = new (std::nothrow) dicegpu_subset_file();
  if (!F) return DICEGPU_ERR_NOMEM;
  try {
    parse(is, width, height, *F);
  } catch (const ParseError& e) {
    if (err && err_len > 0) std::snprintf(err, (size_t)err_len, "%s", e.msg.c_str());
    delete F;
    return DICEGPU_ERR_ARG;
  } catch (...) {
    delete F;
    return DICEGPU_ERR_NOMEM;
  }
  *out = F;
  return DICEGPU_OK;
}

int n_subsets(const dicegpu_subset_file* f) { return (int)(f->coords.size() / 2); }

}  // namespace

extern "C" int dicegpu_subset_file_parse(const char* text, size_t len, int width, int height,
                                         dicegpu_subset_file** out, char* err, int err_len) {
  if (!text || !out) return DICEGPU_ERR_ARG;
  *out = nullptr;
  std::istringstream is(std::string(text, len));
  return finish(is, width, height, out, err, err_len);
}

extern "C" int dicegpu_subset_file_read(const char* path, int width, int height, dicegpu_subset_file** out,
                                        char* err, int err_len) {
  if (!path || !out) return DICEGPU_ERR_ARG;
  *out = nullptr;
  std::ifstream is(path, std::ios::in | std::ios::binary);
  if (!is.good()) {
    if (err && err_len > 0) std::snprintf(err, (size_t)err_len, "the subset file does not exist: %s", path);
    return DICEGPU_ERR_ARG;
  }
  return finish(is, width, height, out, err, err_len);
}

extern "C" int dicegpu_subset_file_free(dicegpu_subset_file* f) {
  delete f;
  return DICEGPU_OK;
}

extern "C" int dicegpu_subset_file_get_info(const dicegpu_subset_file* f, dicegpu_subset_file_info* info) {
  if (!f || !info) return DICEGPU_ERR_ARG;
  std::memset(info, 0, sizeof(*info));
  info->n_subsets = n_subsets(f);
  for (const auto& kv : f->conformal)
    for (const auto& s : kv.second.shapes) {
      ++info->n_shapes;
      info->n_vertices += (int32_t)s.vx.size();
    }
  for (const auto& kv : f->blocking) info->n_blocking_ids += (int32_t)kv.second.size();
  info->n_conformal = (int32_t)f->conformal.size();
  info->region_of_interest = f->roi ? 1 : 0;
  info->n_seeds = (int32_t)f->seeds.size();
  info->n_unsupported = (int32_t)f->features.size();
  info->n_skip_solve_ids = 0;
  for (const auto& kv : f->skip_solve) info->n_skip_solve_ids += (int32_t)kv.second.size();
  return DICEGPU_OK;
}

extern "C" int dicegpu_subset_file_skip_solve(const dicegpu_subset_file* f, uint8_t* has_skip, int32_t* offsets,
                                              int32_t* frame_ids) {
  if (!f || !has_skip || !offsets) return DICEGPU_ERR_ARG;
  const int n = (int)(f->coords.size() / 2);
  int32_t k = 0;
  for (int i = 0; i < n; ++i) {
    offsets[i] = k;
    const auto it = f->skip_solve.find(i);
    has_skip[i] = it != f->skip_solve.end();
    if (has_skip[i]) {
      if (!it->second.empty() && !frame_ids) return DICEGPU_ERR_ARG;
      for (int32_t v : it->second) frame_ids[k++] = v;
    }
  }
  offsets[n] = k;
  return DICEGPU_OK;
}

extern "C" int dicegpu_subset_file_coordinates(const dicegpu_subset_file* f, double* xy) {
  if (!f || (!xy && !f->coords.empty())) return DICEGPU_ERR_ARG;
  std::copy(f->coords.begin(), f->coords.end(), xy);
  return DICEGPU_OK;
}

extern "C" int dicegpu_subset_file_shapes(const dicegpu_subset_file* f, dicegpu_shape* shapes, int32_t* vx,
                                          int32_t* vy) {
  if (!f || !shapes) return DICEGPU_ERR_ARG;
  int k = 0, v = 0;
  for (const auto& kv : f->conformal)
    for (const auto& s : kv.second.shapes) {
      dicegpu_shape o = s.s;
      o.subset = kv.first;
      if (o.kind == DICEGPU_SHAPE_POLYGON) {
        if (!vx || !vy) return DICEGPU_ERR_ARG;
        o.vertex_offset = v;
        for (std::size_t m = 0; m < s.vx.size(); ++m, ++v) { vx[v] = s.vx[m]; vy[v] = s.vy[m]; }
      }
      shapes[k++] = o;
    }
  return DICEGPU_OK;
}

extern "C" int dicegpu_subset_file_blocking(const dicegpu_subset_file* f, int32_t* offsets, int32_t* ids) {
  if (!f || !offsets) return DICEGPU_ERR_ARG;
  const int n = n_subsets(f);
  offsets[0] = 0;
  for (int i = 0; i < n; ++i) {
    const auto it = f->blocking.find(i);
    const int cnt = it == f->blocking.end() ? 0 : (int)it->second.size();
    if (cnt && !ids) return DICEGPU_ERR_ARG;
    for (int m = 0; m < cnt; ++m) ids[offsets[i] + m] = it->second[m];
    offsets[i + 1] = offsets[i] + cnt;
  }
  return DICEGPU_OK;
}

extern "C" int dicegpu_subset_file_force_simplex(const dicegpu_subset_file* f, uint8_t* flags) {
  if (!f || !flags) return DICEGPU_ERR_ARG;
  for (int i = 0; i < n_subsets(f); ++i) flags[i] = f->force_simplex.count(i) ? 1 : 0;
  return DICEGPU_OK;
}

extern "C" int dicegpu_subset_file_seeds(const dicegpu_subset_file* f, double* values, uint8_t* flags) {
  if (!f || !values || !flags) return DICEGPU_ERR_ARG;
  for (int i = 0; i < n_subsets(f); ++i) {
    const auto it = f->seeds.find(i);
    for (int m = 0; m < 6; ++m) values[6 * i + m] = it == f->seeds.end() ? 0.0 : it->second.v[m];
    flags[i] = it == f->seeds.end() ? 0 : (uint8_t)it->second.flags;
  }
  return DICEGPU_OK;
}

extern "C" int dicegpu_subset_file_features(const dicegpu_subset_file* f, uint8_t* flags) {
  if (!f || !flags) return DICEGPU_ERR_ARG;
  for (int i = 0; i < n_subsets(f); ++i) {
    const auto it = f->features.find(i);
    flags[i] = it == f->features.end() ? 0 : (uint8_t)it->second;
  }
  return DICEGPU_OK;
}

namespace {
// Pixel ownership of an undeformed shape (get_owned_pixels,
// DICe_Shape.cpp:136-219, 259-279, 322-420), tested per pixel; the same
// float arithmetic as the device rasterizer, atan2 correctly rounded.
float angle_2d(float x1, float y1, float x2, float y2) {
  const float t1 = (float)std::atan2((double)y1, (double)x1), t2 = (float)std::atan2((double)y2, (double)x2);
  float d = t2 - t1;
  while (d > 3.14159265358979323846) d -= 6.28318530717958647692;
  while (d < -3.14159265358979323846) d += 6.28318530717958647692;
  return d;
}
bool owns(const ShapeDef& d, int x, int y) {
  const dicegpu_shape& s = d.s;
  if (s.kind == DICEGPU_SHAPE_CIRCLE) {
    const int lim = (int)s.radius + 1;
    if (std::abs(x - s.cx) > lim || std::abs(y - s.cy) > lim) return false;
    const float r2 = s.radius * s.radius;
    return (float)((x - s.cx) * (x - s.cx)) + (float)((y - s.cy) * (y - s.cy)) <= r2;
  }
  if (s.kind == DICEGPU_SHAPE_RECTANGLE) {
    const int ox = s.cx - s.width / 2, oy = s.cy - s.height / 2;
    return x >= ox && x < ox + s.width && y >= oy && y < oy + s.height;
  }
  const int nv = (int)d.vx.size();
  float angle = 0.0f;
  for (int i = 0; i < nv; ++i) {
    const int j = (i + 1 == nv) ? 0 : i + 1;
    angle += angle_2d((float)(d.vx[i] - x), (float)(d.vy[i] - y), (float)(d.vx[j] - x), (float)(d.vy[j] - y));
  }
  return std::abs(angle) >= 3.14159265358979323846;
}

// valid_correlation_point (DICe_Decomp.cpp:1070-1120) without the optional
// gradient threshold
bool valid_point(const ConformalDef& roi, int x, int y, int s, int w, int h) {
  if (x < s - 1 || x > w - s || y < s - 1 || y > h - s) return false;
  bool in = false;
  for (const auto& d : roi.shapes)
    if (d.s.role == DICEGPU_ROLE_BOUNDARY && owns(d, x, y)) { in = true; break; }
  if (!in) return false;
  const int cx0 = x - s / 2, cy0 = y - s / 2;
  const int cxs[4] = {cx0, cx0 + s, cx0 + s, cx0}, cys[4] = {cy0, cy0, cy0 + s, cy0 + s};
  for (int k = 0; k < 4; ++k)
    for (const auto& d : roi.shapes)
      if (d.s.role == DICEGPU_ROLE_EXCLUDED && owns(d, cxs[k], cys[k])) return false;
  return true;
}
}  // namespace

extern "C" int dicegpu_regular_grid(const dicegpu_subset_file* f, int width, int height, int step_size,
                                    int subset_size, double* xy, int32_t* neighbor_ids, int32_t* seed_roi,
                                    int cap, int* n_out) {
  if (!n_out || width < 1 || height < 1 || step_size <= 0 || subset_size < 1) return DICEGPU_ERR_ARG;
  if (f && !f->roi) return DICEGPU_ERR_ARG;
  // the regions: the file's, or the whole image (a dummy rectangle ROI)
  std::map<int, ConformalDef> whole;
  const std::map<int, ConformalDef>* rois = f ? &f->conformal : &whole;
  if (!f) {
    ShapeDef d;
    std::memset(&d.s, 0, sizeof(d.s));
    d.s.kind = DICEGPU_SHAPE_RECTANGLE;
    d.s.cx = width / 2;
    d.s.cy = height / 2;
    d.s.width = width;
    d.s.height = height;
    whole[0].shapes.push_back(d);
  }
  const int s = subset_size;
  int n = 0;
  auto push = [&](int x, int y, int neigh, int roi_of_seed) {
    if (n < cap) {
      if (xy) { xy[2 * n] = x; xy[2 * n + 1] = y; }
      if (neighbor_ids) neighbor_ids[n] = neigh;
      if (seed_roi) seed_roi[n] = roi_of_seed;
    }
    ++n;
  };
  for (const auto& kv : *rois) {
    const ConformalDef& roi = kv.second;
    int num_rows = 0, num_cols = 0, seed_row = 0, seed_col = 0, x = s - 1, y = s - 1;
    int seed_x = 0, seed_y = 0;
    bool has_seed = false;
    if (f) {
      const auto it = f->seeds.find(kv.first);
      if (it != f->seeds.end()) { seed_x = it->second.loc_x; seed_y = it->second.loc_y; has_seed = true; }
    }
    while (x < width - s) {
      if (x + step_size / 2 < seed_x) seed_col++;
      x += step_size;
      num_cols++;
    }
    while (y < height - s) {
      if (y + step_size / 2 < seed_y) seed_row++;
      y += step_size;
      num_rows++;
    }
    // the seed point's id is the snakes' first neighbour only when a seed
    // was given (seed_subset_id stays -1 otherwise)
    int seed_id = -1;
    x = s - 1 + seed_col * step_size;
    y = s - 1 + seed_row * step_size;
    if (valid_point(roi, x, y, s, width, height)) {
      if (has_seed) seed_id = n;
      push(x, y, -1, has_seed ? kv.first : -1);
    } else if (!(seed_row == 0 && seed_col == 0)) {
      return DICEGPU_ERR_ARG;   // the seed is not a valid correlation point
    }
    // snake right from the seed, then left
    for (int dir0 = 1; dir0 >= -1; dir0 -= 2) {
      const int start = n;
      int direction = dir0, row = seed_row, col = seed_col;
      while (row >= 0 && row < num_rows) {
        if ((direction == 1 && row + 1 >= num_rows) || (direction == -1 && row - 1 < 0)) {
          direction *= -1;
          col += dir0;
        } else {
          row += direction;
        }
        if (col >= num_cols || col < 0) break;
        x = s - 1 + col * step_size;
        y = s - 1 + row * step_size;
        if (valid_point(roi, x, y, s, width, height)) push(x, y, n == start ? seed_id : n - 1, -1);
      }
    }
  }
  *n_out = n;
  return n <= cap ? DICEGPU_OK : DICEGPU_ERR_ARG;
}

extern "C" int dicegpu_subset_file_apply(const dicegpu_subset_file* f, dicegpu_ctx* ctx) {
  if (!f || !ctx) return DICEGPU_ERR_ARG;
  if (f->roi || !f->features.empty()) return DICEGPU_ERR_UNSUPPORTED;
  dicegpu_params P;
  int rc = dicegpu_get_params(ctx, &P);
  if (rc) return rc;
  const int n = n_subsets(f);
  if (n < 1) return DICEGPU_ERR_ARG;
  for (const auto& kv : f->conformal)
    if (kv.first >= n) return DICEGPU_ERR_ARG;   // a definition for a subset without coordinates
  if ((int)f->conformal.size() < n && P.subset_size < 1) return DICEGPU_ERR_ARG;
  // field rows: coordinates, the shape function's identity, the seeds
  std::vector<double> rows((size_t)n * DICEGPU_FIELD_STRIDE, 0.0);
  for (int i = 0; i < n; ++i) {
    double* r = &rows[(size_t)i * DICEGPU_FIELD_STRIDE];
    r[DICEGPU_F_COORD_X] = f->coords[2 * i];
    r[DICEGPU_F_COORD_Y] = f->coords[2 * i + 1];
    if (P.shape_function == DICEGPU_QUADRATIC_SF) {
      r[DICEGPU_F_QUAD_A] = 1.0;
      r[DICEGPU_F_QUAD_A + 7] = 1.0;
    }
    const auto it = f->seeds.find(i);
    if (it == f->seeds.end()) continue;
    const Seed& s = it->second;
    if ((s.flags & (DICEGPU_SF_SEED_NORMAL_STRAIN | DICEGPU_SF_SEED_SHEAR_STRAIN)) &&
        P.shape_function != DICEGPU_AFFINE_SF)
      return DICEGPU_ERR_ARG;   // seeds can only be used with the affine shape function
    r[DICEGPU_F_DISP_X] = s.v[0];
    r[DICEGPU_F_DISP_Y] = s.v[1];
    if (s.flags & DICEGPU_SF_SEED_NORMAL_STRAIN) {
      r[DICEGPU_F_STRETCH_XX] = s.v[2];
      r[DICEGPU_F_STRETCH_YY] = s.v[3];
    }
    if (s.flags & DICEGPU_SF_SEED_SHEAR_STRAIN) r[DICEGPU_F_SHEAR_XY] = s.v[4];
    if (s.flags & DICEGPU_SF_SEED_ROTATION) r[DICEGPU_F_ROT_Z] = s.v[5];
  }
  if ((rc = dicegpu_set_subsets(ctx, n, rows.data()))) return rc;
  dicegpu_subset_file_info info;
  dicegpu_subset_file_get_info(f, &info);
  if (info.n_shapes > 0) {
    std::vector<dicegpu_shape> shapes(info.n_shapes);
    std::vector<int32_t> vx(std::max(info.n_vertices, 1)), vy(std::max(info.n_vertices, 1));
    if ((rc = dicegpu_subset_file_shapes(f, shapes.data(), vx.data(), vy.data()))) return rc;
    if ((rc = dicegpu_set_subset_shapes(ctx, info.n_shapes, shapes.data(), vx.data(), vy.data()))) return rc;
  }
  if (info.n_blocking_ids > 0) {
    std::vector<int32_t> offs(n + 1), ids(info.n_blocking_ids);
    if ((rc = dicegpu_subset_file_blocking(f, offs.data(), ids.data()))) return rc;
    for (int32_t id : ids)
      if (id < 0 || id >= n) return DICEGPU_ERR_ARG;
    if ((rc = dicegpu_set_blocking(ctx, offs.data(), ids.data()))) return rc;
  }
  if (!f->force_simplex.empty()) {
    std::vector<uint8_t> fl(n);
    dicegpu_subset_file_force_simplex(f, fl.data());
    if ((rc = dicegpu_set_force_simplex(ctx, n, fl.data()))) return rc;
  }
  return DICEGPU_OK;
}

extern "C" int dicegpu_subset_file_apply_grid(const dicegpu_subset_file* f, dicegpu_ctx* ctx, int width,
                                              int height, int step_size) {
  if (!ctx) return DICEGPU_ERR_ARG;
  if (f && (!f->roi || !f->features.empty())) return DICEGPU_ERR_UNSUPPORTED;
  dicegpu_params P;
  int rc = dicegpu_get_params(ctx, &P);
  if (rc) return rc;
  if (P.subset_size < 1) return DICEGPU_ERR_ARG;
  int n = 0;
  rc = dicegpu_regular_grid(f, width, height, step_size, P.subset_size, nullptr, nullptr, nullptr, 0, &n);
  if (rc != DICEGPU_OK && rc != DICEGPU_ERR_ARG) return rc;
  if (n < 1) return DICEGPU_ERR_ARG;
  std::vector<double> xy(2 * (size_t)n);
  std::vector<int32_t> neigh(n), seed_roi(n);
  if ((rc = dicegpu_regular_grid(f, width, height, step_size, P.subset_size, xy.data(), neigh.data(),
                                 seed_roi.data(), n, &n)))
    return rc;
  std::vector<double> rows((size_t)n * DICEGPU_FIELD_STRIDE, 0.0);
  for (int i = 0; i < n; ++i) {
    double* r = &rows[(size_t)i * DICEGPU_FIELD_STRIDE];
    r[DICEGPU_F_COORD_X] = xy[2 * i];
    r[DICEGPU_F_COORD_Y] = xy[2 * i + 1];
    if (P.shape_function == DICEGPU_QUADRATIC_SF) {
      r[DICEGPU_F_QUAD_A] = 1.0;
      r[DICEGPU_F_QUAD_A + 7] = 1.0;
    }
    if (!f || seed_roi[i] < 0) continue;
    // Schema::initialize's seeding (DICe_Schema.cpp:1111-1143)
    const Seed& sd = f->seeds.at(seed_roi[i]);
    if ((sd.flags & (DICEGPU_SF_SEED_NORMAL_STRAIN | DICEGPU_SF_SEED_SHEAR_STRAIN)) &&
        P.shape_function != DICEGPU_AFFINE_SF)
      return DICEGPU_ERR_ARG;
    r[DICEGPU_F_DISP_X] = sd.v[0];
    r[DICEGPU_F_DISP_Y] = sd.v[1];
    if (sd.flags & DICEGPU_SF_SEED_NORMAL_STRAIN) {
      r[DICEGPU_F_STRETCH_XX] = sd.v[2];
      r[DICEGPU_F_STRETCH_YY] = sd.v[3];
    }
    if (sd.flags & DICEGPU_SF_SEED_SHEAR_STRAIN) r[DICEGPU_F_SHEAR_XY] = sd.v[4];
    if (sd.flags & DICEGPU_SF_SEED_ROTATION) r[DICEGPU_F_ROT_Z] = sd.v[5];
  }
  if ((rc = dicegpu_set_subsets(ctx, n, rows.data()))) return rc;
  // NEIGHBOR_ID_FS from the decomposition (DICe_Schema.cpp:1302), for the
  // neighbour initializers
  return dicegpu_set_neighbors(ctx, neigh.data());
}
