// Parameter string parser and detector table (see params.h for the
// reference routines each function follows).
#include "params.h"

#include <cctype>
#include <fstream>
#include <istream>
#include <cmath>
#include <cstdlib>
#include <functional>
#include <unordered_map>

namespace madam {
namespace {

std::string strip(const std::string &s) {
  size_t a = s.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  size_t b = s.find_last_not_of(" \t\r\n");
  return s.substr(a, b - a + 1);
}

// Fortran list-directed input reads the first value; a blank, comma or slash
// ends it.
std::string lead_value(const std::string &v) {
  std::string t = strip(v);
  size_t e = t.find_first_of(" ,/\t");
  return e == std::string::npos ? t : t.substr(0, e);
}

bool as_int(const std::string &v, long &out) {
  std::string t = lead_value(v);
  size_t i = (!t.empty() && (t[0] == '+' || t[0] == '-')) ? 1 : 0;
  if (i >= t.size()) return false;
  for (size_t k = i; k < t.size(); ++k)
    if (!std::isdigit((unsigned char)t[k])) return false;
  out = std::strtol(t.c_str(), nullptr, 10);
  return true;
}

bool as_real(const std::string &v, double &out) {
  std::string t = lead_value(v);
  if (t.empty()) return false;
  for (char &c : t)
    if (c == 'd' || c == 'D') c = 'e';  // Fortran exponent letter
  char *end = nullptr;
  out = std::strtod(t.c_str(), &end);
  return end != t.c_str() && *end == '\0';
}

bool as_logical(const std::string &v, bool &out) {
  std::string t = lead_value(v);
  size_t i = (!t.empty() && t[0] == '.') ? 1 : 0;
  if (i >= t.size()) return false;
  char c = (char)std::toupper((unsigned char)t[i]);
  if (c != 'T' && c != 'F') return false;
  out = (c == 'T');
  return true;
}

// parse_detset (inputparam.f90:375-434): "name : det, det, ..."; a name
// with an empty or "all" member names the full detector set instead
void count_detset(Params &p, const std::string &value, bool nopol) {
  size_t c = value.find(':');
  if (c == std::string::npos)
    fail("Failed to parse: " + strip(value) + " for valid detector set name");
  const std::string name = strip(value.substr(0, c));
  if (name.empty()) fail("Empty detset name");
  Params::DetSet ds;
  ds.name = name;
  ds.nopol = nopol;
  std::string rest = strip(value.substr(c + 1));
  for (;;) {
    size_t k = rest.find(',');
    std::string det = strip(k == std::string::npos ? rest : rest.substr(0, k));
    if (det.empty() || det == "all" || det == "All" || det == "ALL") {
      p.detsets[0].name = name;
      return;
    }
    ds.dets.push_back(det);
    if (k == std::string::npos) break;
    rest = strip(rest.substr(k + 1));
  }
  p.detsets.push_back(ds);
  ++p.ndetset;
}

// parse_survey (inputparam.f90:438-492): "name : start - stop, start - stop";
// a name with no span or "all" names the full data span instead
void count_survey(Params &p, const std::string &value) {
  size_t c = value.find(':');
  if (c == std::string::npos)
    fail("Failed to parse: " + strip(value) + " for valid survey name");
  const std::string name = strip(value.substr(0, c));
  if (name.empty()) fail("Empty survey name");
  Params::Survey sv;
  sv.name = name;
  std::string rest = strip(value.substr(c + 1));
  for (;;) {
    size_t dash = rest.find('-');
    if (dash == std::string::npos) {
      if (rest.empty() || rest == "all" || rest == "All" || rest == "ALL") {
        p.surveys[0].name = name;
        return;
      }
      fail("Failed to parse: " + rest + " for valid survey span marker (-)");
    }
    double a, b;
    if (!as_real(rest.substr(0, dash), a))
      fail("Failed to parse: " + rest + " for valid survey start");
    rest = strip(rest.substr(dash + 1));
    if (!as_real(rest, b)) fail("Failed to parse: " + rest + " for valid survey stop");
    sv.starts.push_back(a);
    sv.stops.push_back(b);
    size_t k = rest.find(',');
    if (k == std::string::npos) break;
    rest = strip(rest.substr(k + 1));
  }
  p.surveys.push_back(sv);
  ++p.nsurvey;
}

using Setter = std::function<bool(Params &, const std::string &)>;

Setter I(long Params::*m) {
  return [m](Params &p, const std::string &v) { return as_int(v, p.*m); };
}
Setter D(double Params::*m) {
  return [m](Params &p, const std::string &v) { return as_real(v, p.*m); };
}
Setter L(bool Params::*m) {
  return [m](Params &p, const std::string &v) { return as_logical(v, p.*m); };
}
Setter S(std::string Params::*m) {
  return [m](Params &p, const std::string &v) { p.*m = strip(v); return true; };
}

const std::unordered_map<std::string, Setter> &keytable() {
  static const std::unordered_map<std::string, Setter> t = {
      {"info", I(&Params::info)},
      {"nthreads", I(&Params::nthreads)},
      {"nsubchunk", I(&Params::nsubchunk)},
      {"isubchunk", I(&Params::isubchunk)},
      {"time_unit",
       [](Params &p, const std::string &v) {
         std::string s = strip(v);
         if (!s.empty() && (s[0] == 'p' || s[0] == 'P')) { p.time_unit = -5; return true; }
         return as_real(v, p.time_unit);
       }},
      {"base_first", D(&Params::dnshort)},
      {"nshort", D(&Params::dnshort)},
      {"nside_map", I(&Params::nside_map)},
      {"nside_cross", I(&Params::nside_cross)},
      {"nside_submap", I(&Params::nside_submap)},
      {"good_baseline_fraction", D(&Params::good_baseline_fraction)},
      {"concatenate_messages", L(&Params::concatenate_messages)},
      {"allreduce", L(&Params::allreduce)},
      {"reassign_submaps", L(&Params::reassign_submaps)},
      {"pixmode_map", I(&Params::pixmode_map)},
      {"pixmode_cross", I(&Params::pixmode_cross)},
      {"pixlim_map", D(&Params::pixlim_map)},
      {"pixlim_cross", D(&Params::pixlim_cross)},
      {"incomplete_matrices", L(&Params::incomplete_matrices)},
      {"allow_decoupling", L(&Params::allow_decoupling)},
      {"kfirst", L(&Params::kfirst)},
      {"basis_func",
       [](Params &p, const std::string &v) {
         std::string s = strip(v).substr(0, 4);
         if (s == "poly") p.basis_func = 1;
         else if (s == "four") p.basis_func = 2;
         else if (s == "cheb") p.basis_func = 3;
         else if (s == "lege") p.basis_func = 4;
         else fail("Unknown function basis : " + strip(v));
         return true;
       }},
      {"basis_order",
       [](Params &p, const std::string &v) {
         if (!as_int(v, p.basis_order)) return false;
         if (p.basis_order < 0) fail("basis order must be nonnegative");
         return true;
       }},
      {"iter_min", I(&Params::iter_min)},
      {"iter_max", I(&Params::iter_max)},
      {"cglimit", D(&Params::cglimit)},
      {"fsample", D(&Params::fsample)},
      {"mode_detweight", I(&Params::mode_detweight)},
      {"flag_by_horn", L(&Params::flag_by_horn)},
      {"write_cut", L(&Params::write_cut)},
      {"checknan", L(&Params::checknan)},
      {"sync_output", L(&Params::sync_output)},
      {"skip_existing", L(&Params::skip_existing)},
      {"temperature_only", L(&Params::temperature_only)},
      {"force_pol", L(&Params::force_pol)},
      {"noise_weights_from_psd", L(&Params::noise_weights_from_psd)},
      {"radiometers", L(&Params::radiometers)},
      {"psdlen", I(&Params::psdlen)},
      {"psd_down", I(&Params::psd_downsample)},
      {"psd_downsample", I(&Params::psd_downsample)},
      {"kfilter", L(&Params::kfilter)},
      {"diagfilter", D(&Params::diagfilter)},
      {"unaligned_fft", L(&Params::unaligned_fft)},
      {"precond_width_min", I(&Params::precond_width_min)},
      {"precond_width_max", I(&Params::precond_width_max)},
      {"use_fprecond", L(&Params::use_fprecond)},
      {"use_cgprecond", L(&Params::use_cgprecond)},
      {"rm_monopole", L(&Params::rm_monopole)},
      {"path_output", S(&Params::path_output)},
      {"file_root", S(&Params::file_root)},
      {"write_map", L(&Params::do_map)},
      {"write_binmap", L(&Params::do_binmap)},
      {"write_hits", L(&Params::do_hits)},
      {"write_matrix", L(&Params::do_matrix)},
      {"write_wcov", L(&Params::do_wcov)},
      {"write_base", L(&Params::do_base)},
      {"write_mask", L(&Params::do_mask)},
      {"write_leakmatrix", L(&Params::do_leakmatrix)},
      {"unit_tod", S(&Params::unit_tod)},
      {"file_gap_out", S(&Params::file_gap_out)},
      {"file_mc", S(&Params::file_mc)},
      {"write_tod", L(&Params::write_tod)},
      {"file_inmask", S(&Params::file_inmask)},
      {"file_spectrum", S(&Params::file_spectrum)},
      {"file_gap", S(&Params::file_gap)},
      {"binary_output", L(&Params::binary_output)},
      {"nwrite_binary", I(&Params::nwrite_binary)},
      {"file_covmat", S(&Params::file_covmat)},
      {"detset", [](Params &p, const std::string &v) { count_detset(p, v, false); return true; }},
      {"detset_nopol",
       [](Params &p, const std::string &v) { count_detset(p, v, true); return true; }},
      {"survey", [](Params &p, const std::string &v) { count_survey(p, v); return true; }},
      {"bin_subsets", L(&Params::bin_subsets)},
      {"mcmode", L(&Params::mcmode)},
  };
  return t;
}

void apply_line(Params &p, const std::string &raw) {
  std::string line = strip(raw);
  if (line.empty()) return;
  size_t eq = line.find('=');
  if (line[0] == '#') return;
  if (eq == std::string::npos) fail("Syntax error in parameter definition: " + line);
  std::string key = strip(line.substr(0, eq)).substr(0, 40);
  std::string value = strip(line.substr(eq + 1)).substr(0, 200);
  size_t hash = value.find('#');
  if (hash != std::string::npos) value.resize(hash);
  if (key.compare(0, 8, "detector") == 0) key = "detector";
  if (strip(value).empty() && key.compare(0, 4, "file") != 0) return;
  auto it = keytable().find(key);
  if (it == keytable().end()) fail("Unknown parameter: " + key);
  if (!it->second(p, value)) fail("Failed to parse " + key + " from " + strip(value));
}

}  // namespace

Params parse_parstring(const char *parstring) {
  Params p;
  std::string s(parstring ? parstring : "");
  size_t pos = 0;
  while (pos < s.size()) {
    size_t semi = s.find(';', pos);
    if (semi == std::string::npos) semi = s.size();
    apply_line(p, s.substr(pos, semi - pos));
    pos = semi + 1;
  }
  p.dnshort = std::round(p.dnshort * p.fsample);  // nint(): half away from zero
  if (p.kfirst && p.dnshort < 0) p.dnshort = 1e10;
  return p;
}

std::vector<Detector> read_detectors(const Params &p, const char *detstring,
                                     long ndet, const double *detweights,
                                     const long *npsd, long npsdtot,
                                     const double *psdstarts, long npsdbin,
                                     const double *psdfreqs, long npsdval,
                                     const double *psdvals) {
  std::vector<Detector> dets(ndet);
  std::string s(detstring ? detstring : "");
  size_t pos = 0;
  long idet = 0, ipsd = 0, off = 0;
  while (pos < s.size()) {
    size_t semi = s.find(';', pos);
    if (semi == std::string::npos) semi = s.size();
    if (idet >= ndet) fail("Too many detectors");
    Detector &d = dets[idet];
    d.name = strip(s.substr(pos, semi - pos)).substr(0, 20);
    long nint = npsd[idet];
    d.npsd = nint == 0 ? 1 : (int)nint;
    double w = detweights[idet];
    d.weights.assign(d.npsd, w);
    d.sigmas.assign(d.npsd, w > 0 ? 1.0 / std::sqrt(w) : 0.0);
    d.plateaus.resize(d.npsd);
    for (int i = 0; i < d.npsd; ++i) d.plateaus[i] = d.sigmas[i] * d.sigmas[i] / p.fsample;
    d.psdstarts.assign(d.npsd, 0.0);
    if (nint > 0) {
      d.has_psd = true;
      d.psdfreqs.assign(psdfreqs, psdfreqs + npsdbin);
      d.psds.assign(nint, std::vector<double>(npsdbin));
      for (long i = 0; i < nint; ++i) {
        if (ipsd >= npsdtot || off + npsdbin > npsdval) fail("PSD arrays are too short");
        d.psdstarts[i] = psdstarts[ipsd++];
        for (long b = 0; b < npsdbin; ++b) d.psds[i][b] = psdvals[off + b];
        off += npsdbin;
      }
    }
    ++idet;
    pos = semi + 1;
  }
  return dets;
}

void interpolate_psd(const std::vector<double> &freq,
                     const std::vector<double> &psd, const double *target,
                     double *out, long nout) {
  const long nin = (long)freq.size();
  if ((long)psd.size() != nin) fail("freq and psd do not have the same shape");
  long first = 0;
  while (first < nin && freq[first] == 0) ++first;
  if (first == nin) fail("input freqs are all zero.");
  std::vector<double> lf(nin), lp(nin);
  for (long i = 0; i < nin; ++i) {
    lf[i] = std::log(freq[i]);
    lp[i] = std::log(psd[i]);
  }
  long j = first;
  for (long i = 0; i < nout; ++i) {
    if (target[i] == 0) {
      out[i] = 0;
      continue;
    }
    const double flog = std::log(target[i]);
    if (j < nin - 2) {
      while (lf[j + 1] < flog) {
        if (++j == nin - 2) break;
      }
    }
    if (psd[j] > 0 && psd[j + 1] > 0) {
      const double r = (flog - lf[j]) / (lf[j + 1] - lf[j]);
      out[i] = std::exp(lp[j] * (1.0 - r) + lp[j + 1] * r);
    } else {
      const double r = (target[i] - freq[j]) / (freq[j + 1] - freq[j]);
      out[i] = psd[j] * (1.0 - r) + psd[j + 1] * r;
    }
  }
}

int psd_index_det(const Detector &d, double t) {
  if (!d.has_psd && d.npsd == 1) return 0;
  for (int i = 0;; ++i) {
    if (i == d.npsd - 1) return d.psdstarts[i] > t ? -1 : i;
    if (d.psdstarts[i + 1] > t) return i;
  }
}

}  // namespace madam

namespace madam {

namespace {

// Fortran list-directed input: every READ starts at a new record, takes its
// items from as many records as it needs (separated by blanks or commas,
// strings possibly quoted) and drops the rest of the last record it used.
class ListInput {
 public:
  explicit ListInput(std::istream &in) {
    std::string line;
    while (std::getline(in, line)) lines_.push_back(line);
  }
  // n items of one READ; false at the end of the file, and where the READ
  // would leave items undefined: a null value ("r*" with no constant) or a
  // slash that ends the READ early
  bool read(size_t n, std::vector<std::string> &out) {
    out.clear();
    while (out.size() < n) {
      if (rec_ >= lines_.size()) return false;
      if (!split(lines_[rec_++], out, n)) return false;
    }
    return true;
  }

 private:
  static bool split(const std::string &s, std::vector<std::string> &out, size_t n) {
    size_t i = 0;
    while (i < s.size() && out.size() < n) {
      while (i < s.size() && (std::isspace((unsigned char)s[i]) || s[i] == ',')) ++i;
      if (i >= s.size()) break;
      if (s[i] == '/') return false;
      // a repeat count "r*c": r copies of the constant c
      size_t r = 1, j = i;
      while (j < s.size() && std::isdigit((unsigned char)s[j])) ++j;
      if (j > i && j < s.size() && s[j] == '*') {
        if (j - i > 9) return false;
        r = std::stoul(s.substr(i, j - i));
        i = j + 1;
        if (r == 0 || i >= s.size() || std::isspace((unsigned char)s[i]) || s[i] == ',')
          return false;
      }
      std::string tok;
      if (s[i] == '\'' || s[i] == '"') {
        const char q = s[i++];
        while (i < s.size()) {
          if (s[i] == q) {
            if (i + 1 < s.size() && s[i + 1] == q) {
              tok += q;
              i += 2;
              continue;
            }
            ++i;
            break;
          }
          tok += s[i++];
        }
      } else {
        while (i < s.size() && !std::isspace((unsigned char)s[i]) && s[i] != ',') tok += s[i++];
      }
      for (size_t k = 0; k < r && out.size() < n; ++k) out.push_back(tok);
    }
    return true;
  }
  std::vector<std::string> lines_;
  size_t rec_ = 0;
};

bool to_real(std::string t, double &v) {
  for (char &c : t)
    if (c == 'd' || c == 'D') c = 'e';
  char *end = nullptr;
  v = std::strtod(t.c_str(), &end);
  return end && *end == '\0' && !t.empty();
}

bool to_reals(const std::vector<std::string> &tok, std::vector<double> &v) {
  v.resize(tok.size());
  for (size_t i = 0; i < tok.size(); ++i)
    if (!to_real(tok[i], v[i])) return false;
  return true;
}

}  // namespace

SpectrumFile read_spectrum_file(const std::string &path, const std::vector<Detector> &dets) {
  // read_spectrum (noise_routines.f90:505-596): "nobins nodetectors", the
  // detector names, their sigmas, then one row "freq psd_1 .. psd_n" per bin
  std::ifstream f(path);
  if (!f) fail("ERROR, cannot open " + path);
  ListInput in(f);
  std::vector<std::string> tok;
  std::vector<double> v;
  if (!in.read(2, tok) || !to_reals(tok, v) || v[0] < 2 || v[1] < 1 || v[0] != (long)v[0] ||
      v[1] != (long)v[1])
    fail("ERROR, " + path + " is not formatted correctly");
  const long nolines = (long)v[0], nocols = (long)v[1];
  std::vector<std::string> names;
  if (!in.read((size_t)nocols, names))
    fail("Failed to read detector names from spectrum file");
  std::vector<double> sig;
  if (!in.read((size_t)nocols, tok) || !to_reals(tok, sig))
    fail("Failed to read detector noise levels from spectrum file");
  std::vector<double> tab;
  if (!in.read((size_t)(nocols + 1) * nolines, tok) || !to_reals(tok, tab))
    fail("Failed to read the table from spectrum file");
  SpectrumFile sf;
  sf.logf.resize(nolines);
  for (long l = 0; l < nolines; ++l) sf.logf[l] = std::log(tab[(size_t)l * (nocols + 1)]);
  for (const Detector &d : dets) {
    long icol = 0;
    while (icol < nocols && names[icol].find(d.name) == std::string::npos) ++icol;
    if (icol == nocols) fail("ERROR: " + d.name + " not in " + path);
    sf.sigma.push_back(sig[icol]);
    std::vector<double> ls(nolines);
    for (long l = 0; l < nolines; ++l)
      ls[l] = std::log(tab[(size_t)l * (nocols + 1) + 1 + icol]);
    sf.logspec.push_back(std::move(ls));
  }
  return sf;
}

void spectrum_from_file(const SpectrumFile &sf, int idet, const double *f, double *out,
                        long nout) {
  const std::vector<double> &ft = sf.logf, &st = sf.logspec[idet];
  const long nl = (long)ft.size();
  long k = 0;
  for (long i = 0; i < nout; ++i) {
    const double logf = std::log(f[i]);
    while (!(logf <= ft[k + 1] || k == nl - 2)) ++k;
    double p = (logf - ft[k]) / (ft[k + 1] - ft[k]);
    if (p < 0) p = 0;
    if (p > 1) p = 1;
    out[i] = std::exp((1.0 - p) * st[k] + p * st[k + 1]);
  }
}

}  // namespace madam
