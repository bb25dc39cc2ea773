// config.cpp -- Utilities::ConfigFile (Config.h:21-85, Config.cpp:11-300) as a
// C entry point, with the reference's keyword file format:
//
//   # comment
//   GridDimension   NumX NumY NumZ
//   InputStrainRate
//     s00 s01 s02          (three continuation lines, rows of the 3x3 matrix)
//     s10 s11 s12
//     s20 s21 s22
//   MaxNRIter       n
//   TimeStep        dt
//   NumTimeIter     n
//   NRTolerence     eps
//   TwoGrainInit  |  FileInit <filename>
//   CRSS            12 values (or 1, applied to all systems)
//   GammaDotBase    12 values (or 1)
//   RateSensitivity 12 values (or 1)
//
// Keywords added for the material and solver constants the reference
// hard-codes (MaterialGrid.cpp:322-336, 390, 445): Tau0, Tau1, Theta0,
// Theta1 (12 values or 1), HardeningMatrix (144 values or 1, may continue on
// following indented lines), VoxelLength hx hy hz, ConvergenceEpsilon e, MaxIter n,
// Precision FP64|MIXED.
//
// Defects of the reference that are not reproduced: slip-system values are
// stored at indices 0..11 (it writes 1..12 into size-12 vectors,
// Config.cpp:195-197, 203-205, 211-213); Parse returns its result (it falls
// off the end, Config.cpp:261); continuation lines are recognised by not
// starting with a keyword (Config.h:77 used find_first_of); NRTolerence and
// TimeStep are double (Config.h:39-40); errors are returned, never exit().
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/vpfft_capi.h"

namespace {

const char* const kKeywords[] = {"GridDimension", "InputStrainRate", "MaxNRIter",     "TimeStep",
                                 "NumTimeIter",   "NRTolerence",     "TwoGrainInit",  "FileInit",
                                 "CRSS",          "GammaDotBase",    "RateSensitivity", "Tau0",
                                 "Tau1",          "Theta0",          "Theta1",        "HardeningMatrix",
                                 "VoxelLength",   "ConvergenceEpsilon", "MaxIter",    "Precision"};
constexpr int kNumKeywords = sizeof(kKeywords) / sizeof(kKeywords[0]);

bool is_keyword(const std::string& t) {
  for (int k = 0; k < kNumKeywords; ++k)
    if (t == kKeywords[k]) return true;
  return false;
}

bool to_double(const std::string& s, double* v) {
  char* end = nullptr;
  *v = std::strtod(s.c_str(), &end);
  return end && *end == '\0' && !s.empty();
}
bool to_int(const std::string& s, int* v) {
  char* end = nullptr;
  long x = std::strtol(s.c_str(), &end, 10);
  if (!end || *end != '\0' || s.empty()) return false;
  *v = (int)x;
  return true;
}

struct Parser {
  std::vector<std::vector<std::string>> lines;
  std::vector<bool> indented;  // line starts with white space: a continuation line
  std::string err;
  bool fail(size_t line, const std::string& m) {
    err = "line " + std::to_string(line + 1) + ": " + m;
    return false;
  }
};

}  // namespace

extern "C" vpfft_status vpfft_config_read(const char* path, vpfft_config* out, char* err,
                                          size_t err_len) {
  auto set_err = [&](const std::string& m) {
    if (err && err_len) {
      std::snprintf(err, err_len, "%s", m.c_str());
    }
  };
  if (!path || !out) {
    set_err("NULL argument");
    return VPFFT_ERR_INVALID_ARGUMENT;
  }
  std::ifstream f(path);
  if (!f) {
    set_err(std::string("cannot open ") + path);
    return VPFFT_ERR_IO;
  }
  std::memset(out, 0, sizeof(*out));
  vpfft_material_default(&out->material);
  out->voxel_length[0] = out->voxel_length[1] = out->voxel_length[2] = 1.0;
  out->convergence_epsilon = 1e-5;
  out->max_iter = 100;
  out->precision = VPFFT_PREC_FP64;
  out->init_method = -1;

  Parser P;
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream is(line);
    std::vector<std::string> toks;
    std::string t;
    while (is >> t) toks.push_back(t);
    P.lines.push_back(toks);
    P.indented.push_back(!line.empty() && (line[0] == ' ' || line[0] == '\t'));
  }
  bool seen[kNumKeywords] = {false};
  auto seen_kw = [&](const char* k) {
    for (int i = 0; i < kNumKeywords; ++i)
      if (!std::strcmp(kKeywords[i], k)) return seen[i];
    return false;
  };
  // values of a keyword: the rest of its line plus the following continuation
  // lines (indented, not starting with a keyword or a comment)
  auto gather = [&](size_t& i) {
    std::vector<std::string> v(P.lines[i].begin() + 1, P.lines[i].end());
    while (i + 1 < P.lines.size() && !P.lines[i + 1].empty() && P.indented[i + 1] &&
           !is_keyword(P.lines[i + 1][0]) && P.lines[i + 1][0][0] != '#') {
      ++i;
      v.insert(v.end(), P.lines[i].begin(), P.lines[i].end());
    }
    return v;
  };
  auto per_system = [&](size_t i, const std::vector<std::string>& v, double* dst, int count,
                        const char* name) -> bool {
    if ((int)v.size() != count && v.size() != 1)
      return P.fail(i, std::string(name) + ": expected " + std::to_string(count) + " values or 1");
    for (int k = 0; k < count; ++k) {
      double x;
      if (!to_double(v[v.size() == 1 ? 0 : k], &x)) return P.fail(i, std::string(name) + ": bad number");
      dst[k] = x;
    }
    return true;
  };

  bool ok = true;
  for (size_t i = 0; ok && i < P.lines.size(); ++i) {
    const auto& L = P.lines[i];
    if (L.empty() || L[0][0] == '#') continue;
    const std::string& kw = L[0];
    int id = -1;
    for (int k = 0; k < kNumKeywords; ++k)
      if (kw == kKeywords[k]) id = k;
    if (id < 0) {
      ok = P.fail(i, "syntax not recognized: " + kw);
      break;
    }
    seen[id] = true;
    const size_t line0 = i;
    std::vector<std::string> v = gather(i);
    if (kw == "GridDimension") {
      if (v.size() != 3 || !to_int(v[0], &out->num_x) || !to_int(v[1], &out->num_y) ||
          !to_int(v[2], &out->num_z))
        ok = P.fail(line0, "GridDimension: expected 3 integers [NumX NumY NumZ]");
    } else if (kw == "InputStrainRate") {
      if (v.size() != 9) {
        ok = P.fail(line0, "InputStrainRate: expected 3 continuation lines of 3 numbers");
      } else {
        for (int k = 0; k < 9 && ok; ++k)
          if (!to_double(v[k], &out->input_strain_rate[k])) ok = P.fail(line0, "InputStrainRate: bad number");
      }
    } else if (kw == "MaxNRIter") {
      if (v.size() != 1 || !to_int(v[0], &out->max_nr_iter)) ok = P.fail(line0, "MaxNRIter: expected an integer");
    } else if (kw == "TimeStep") {
      if (v.size() != 1 || !to_double(v[0], &out->time_step)) ok = P.fail(line0, "TimeStep: expected a number");
    } else if (kw == "NumTimeIter") {
      if (v.size() != 1 || !to_int(v[0], &out->num_time_iter)) ok = P.fail(line0, "NumTimeIter: expected an integer");
    } else if (kw == "NRTolerence") {
      if (v.size() != 1 || !to_double(v[0], &out->nr_tolerance)) ok = P.fail(line0, "NRTolerence: expected a number");
    } else if (kw == "TwoGrainInit") {
      out->init_method = 0;
    } else if (kw == "FileInit") {
      if (v.size() != 1) {
        ok = P.fail(line0, "FileInit: expect filename for initialization");
      } else {
        std::snprintf(out->input_microstructure, sizeof(out->input_microstructure), "%s", v[0].c_str());
        std::ifstream probe(v[0]);
        if (!probe) ok = P.fail(line0, "FileInit " + v[0] + " not found");
        out->init_method = 1;
      }
    } else if (kw == "CRSS") {
      ok = per_system(line0, v, out->material.crss, 12, "CRSS");
    } else if (kw == "GammaDotBase") {
      ok = per_system(line0, v, out->material.gamma_dot_base, 12, "GammaDotBase");
    } else if (kw == "RateSensitivity") {
      double tmp[12];
      ok = per_system(line0, v, tmp, 12, "RateSensitivity");
      for (int k = 0; ok && k < 12; ++k) {
        out->material.rate_sensitivity[k] = (int32_t)tmp[k];
        if ((double)out->material.rate_sensitivity[k] != tmp[k]) ok = P.fail(line0, "RateSensitivity: integers expected");
      }
    } else if (kw == "Tau0") {
      ok = per_system(line0, v, out->material.tau0, 12, "Tau0");
    } else if (kw == "Tau1") {
      ok = per_system(line0, v, out->material.tau1, 12, "Tau1");
    } else if (kw == "Theta0") {
      ok = per_system(line0, v, out->material.theta0, 12, "Theta0");
    } else if (kw == "Theta1") {
      ok = per_system(line0, v, out->material.theta1, 12, "Theta1");
    } else if (kw == "HardeningMatrix") {
      ok = per_system(line0, v, out->material.hardening, 144, "HardeningMatrix");
    } else if (kw == "VoxelLength") {
      if (v.size() != 3) ok = P.fail(line0, "VoxelLength: expected 3 numbers");
      for (int k = 0; ok && k < 3; ++k)
        if (!to_double(v[k], &out->voxel_length[k]) || !(out->voxel_length[k] > 0))
          ok = P.fail(line0, "VoxelLength: positive numbers expected");
    } else if (kw == "ConvergenceEpsilon") {
      if (v.size() != 1 || !to_double(v[0], &out->convergence_epsilon))
        ok = P.fail(line0, "ConvergenceEpsilon: expected a number");
    } else if (kw == "MaxIter") {
      if (v.size() != 1 || !to_int(v[0], &out->max_iter)) ok = P.fail(line0, "MaxIter: expected an integer");
    } else if (kw == "Precision") {
      if (v.size() == 1 && v[0] == "FP64")
        out->precision = VPFFT_PREC_FP64;
      else if (v.size() == 1 && v[0] == "MIXED")
        out->precision = VPFFT_PREC_MIXED;
      else
        ok = P.fail(line0, "Precision: FP64 or MIXED");
    }
  }
  if (ok) {
    // required keywords of the reference (Config.cpp:178-184, 314-329)
    const char* req[] = {"GridDimension", "InputStrainRate", "MaxNRIter", "TimeStep", "NumTimeIter",
                         "NRTolerence",   "CRSS",            "GammaDotBase", "RateSensitivity"};
    for (const char* r : req)
      if (ok && !seen_kw(r)) {
        P.err = std::string("missing parameter: ") + r + " not optional";
        ok = false;
      }
    if (ok && out->init_method < 0) {
      P.err = "initialization scheme (either FileInit or TwoGrainInit) needs to be specified";
      ok = false;
    }
  }
  if (!ok) {
    set_err(P.err);
    return VPFFT_ERR_IO;
  }
  set_err("");
  return VPFFT_OK;
}
