// FITS products of destripe(): HEALPix binary tables like the reference's
// output.f90 (write_map 114-375, write_binmap 526-786, write_mask 792-912,
// write_hits 918-1025, write_matrix 1031-1175, headers 1376-1591).
//
// Layout (full sky, NESTED): one row per submap, one column per map
// component with nosubpix values per row ('E' float32 maps, 'J' hits and
// mask, 'D' pixel matrices); unobserved map pixels hold the HEALPix
// undefined value -1.6375e30.  Files are named <path_output><file_root>
// _map.fits, _bmap.fits, _hmap.fits, _mask.fits, _wcov_inv.fits, _wcov.fits,
// _leakmatrix_<detector>.fits (write_leakmatrix 1181-1323), and the subset
// products of run_subsets (smadam.F90:954-1257);
// an existing file gets a _001, _002, ... suffix unless the name starts with
// '!' (check_outfile, output.f90:1329-1366).
#include "fits.h"

#include <sys/stat.h>

#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace madam {
namespace {

const float kUndef = -1.6375e30f;

bool exists(const std::string &f) {
  struct stat st;
  return stat(f.c_str(), &st) == 0;
}

std::string resolve(std::string f) {
  if (!f.empty() && f[0] == '!') return f.substr(1);
  if (!exists(f)) return f;
  const size_t dot = f.rfind('.');
  const std::string stem = dot == std::string::npos ? f : f.substr(0, dot);
  const std::string ext = dot == std::string::npos ? "" : f.substr(dot);
  for (int k = 1; k < 1000; ++k) {
    char s[8];
    std::snprintf(s, sizeof s, "_%03d", k);
    const std::string c = stem + s + ext;
    if (!exists(c)) return c;
  }
  return "";
}

class Header {
 public:
  void raw(const std::string &c) {
    std::string s = c.substr(0, 80);
    s.resize(80, ' ');
    cards_.push_back(s);
  }
  void str(const std::string &k, const std::string &v, const std::string &cm = "") {
    std::string q = "'" + v;
    while (q.size() < 9) q += ' ';
    q += "'";
    kv(k, q, cm, false);
  }
  void integer(const std::string &k, long long v, const std::string &cm = "") {
    kv(k, std::to_string(v), cm, true);
  }
  void real(const std::string &k, double v, const std::string &cm = "") {
    char b[32];
    std::snprintf(b, sizeof b, "%.10E", v);
    kv(k, b, cm, true);
  }
  void logical(const std::string &k, bool v, const std::string &cm = "") {
    kv(k, v ? "T" : "F", cm, true);
  }
  void comment(const std::string &t) { raw("COMMENT " + t); }
  void write(FILE *f) {
    raw("END");
    for (auto &c : cards_) std::fwrite(c.data(), 1, 80, f);
    const size_t n = cards_.size() * 80;
    const size_t pad = (2880 - n % 2880) % 2880;
    std::string sp(pad, ' ');
    std::fwrite(sp.data(), 1, pad, f);
    cards_.clear();
  }

 private:
  void kv(const std::string &k, const std::string &v, const std::string &cm, bool right) {
    std::string key = k;
    for (auto &ch : key) ch = (char)toupper(ch);
    key.resize(8, ' ');
    std::string val = v;
    if (right && val.size() < 20) val = std::string(20 - val.size(), ' ') + val;
    std::string c = key + "= " + val;
    if (!cm.empty()) c += " / " + cm;
    raw(c);
  }
  std::vector<std::string> cards_;
};

template <typename T>
void put_be(std::vector<unsigned char> &out, T v) {
  unsigned char b[sizeof(T)];
  std::memcpy(b, &v, sizeof(T));
  for (int i = (int)sizeof(T) - 1; i >= 0; --i) out.push_back(b[i]);
}

struct Col {
  std::string name, tform, unit;
  int bytes;  // per row
};

// One BINTABLE file: empty primary HDU + table.  row(r, buf) appends row r.
template <typename KeyFn, typename RowFn>
void write_table(const std::string &fname, const std::vector<Col> &cols, long long nrows,
                 KeyFn keys, RowFn row) {
  FILE *f = std::fopen(fname.c_str(), "wb");
  if (!f) fail("cannot open " + fname + " for writing");
  Header p;
  p.logical("SIMPLE", true, "file does conform to FITS standard");
  p.integer("BITPIX", 8, "number of bits per data pixel");
  p.integer("NAXIS", 0, "number of data axes");
  p.logical("EXTEND", true, "FITS dataset may contain extensions");
  p.write(f);
  long long rowbytes = 0;
  for (auto &c : cols) rowbytes += c.bytes;
  Header h;
  h.str("XTENSION", "BINTABLE", "binary table extension");
  h.integer("BITPIX", 8, "8-bit bytes");
  h.integer("NAXIS", 2, "2-dimensional binary table");
  h.integer("NAXIS1", rowbytes, "width of table in bytes");
  h.integer("NAXIS2", nrows, "number of rows in table");
  h.integer("PCOUNT", 0, "size of special data area");
  h.integer("GCOUNT", 1, "one data group (required keyword)");
  h.integer("TFIELDS", (long long)cols.size(), "number of fields in each row");
  for (size_t i = 0; i < cols.size(); ++i) {
    const std::string n = std::to_string(i + 1);
    h.str("TTYPE" + n, cols[i].name, "label for field");
    h.str("TFORM" + n, cols[i].tform, "data format of field");
    if (!cols[i].unit.empty()) h.str("TUNIT" + n, cols[i].unit, "physical unit of field");
  }
  keys(h);
  std::vector<unsigned char> buf;
  h.write(f);
  long long total = 0;
  for (long long r = 0; r < nrows; ++r) {
    buf.clear();
    row(r, buf);
    std::fwrite(buf.data(), 1, buf.size(), f);
    total += (long long)buf.size();
  }
  const long long pad = (2880 - total % 2880) % 2880;
  std::vector<unsigned char> z(pad, 0);
  std::fwrite(z.data(), 1, pad, f);
  std::fclose(f);
}

// HEALPix tables of one run (or one subset of it): full-sky host arrays at
// nside_map with nmap components.
class Tables {
 public:
  Tables(const Params &p, long nsub, long nsm, long ndet, int nmap)
      : p_(p), nsub_(nsub), nsm_(nsm), ndet_(ndet), nmap_(nmap) {}

  void map(const std::string &f, const double *m, const int *mask, const char *objtype) {
    if (f.empty()) return;
    const char *mapnames[3] = {"TEMPERATURE", "Q-POLARISATION", "U-POLARISATION"};
    std::vector<Col> cols;
    for (int j = 0; j < nmap_; ++j)
      cols.push_back({nmap_ == 3 ? mapnames[j] : "TEMPERATURE", std::to_string(nsub_) + "E",
                      p_.unit_tod, (int)(4 * nsub_)});
    auto keys = [&](Header &h) {
      h.str("OBJTYPE", objtype, "Object type");
      healpix(h);
      h.logical("MONOPOLE", p_.rm_monopole, "Monopole removed (T map)");
    };
    write_table(f, cols, nsm_, keys, [&](long long r, std::vector<unsigned char> &b) {
      for (int j = 0; j < nmap_; ++j)
        for (long i = 0; i < nsub_; ++i) {
          const long px = r * nsub_ + i;
          const float v = mask[px] > 0 ? (float)m[px * nmap_ + j] : kUndef;
          put_be(b, v);
        }
    });
  }

  void hits(const std::string &f, const int *hits) {
    if (f.empty()) return;
    const long npix = nsub_ * nsm_;
    long rep = std::max<long>(12 * 1024, nsub_);
    rep = std::min<long>(rep, npix);
    const long nrows = (npix + rep - 1) / rep;
    std::vector<Col> cols = {{"Total hits", std::to_string(rep) + "J", "", (int)(4 * rep)}};
    auto keys = [&](Header &h) {
      h.str("OBJTYPE", "madam.hits", "Object type");
      healpix(h);
    };
    write_table(f, cols, nrows, keys, [&](long long r, std::vector<unsigned char> &b) {
      for (long i = 0; i < rep; ++i) {
        const long px = r * rep + i;
        put_be(b, (int32_t)(px < npix ? hits[px] : 0));
      }
    });
  }

  void mask(const std::string &f, const int *mask, const float *crit) {
    if (f.empty()) return;
    std::vector<Col> cols = {{"Mask", std::to_string(nsub_) + "J", "", (int)(4 * nsub_)},
                             {"criterion", std::to_string(nsub_) + "E", "", (int)(4 * nsub_)}};
    auto keys = [&](Header &h) {
      h.str("OBJTYPE", "madam.mask", "Object type");
      healpix(h);
    };
    write_table(f, cols, nsm_, keys, [&](long long r, std::vector<unsigned char> &b) {
      for (long i = 0; i < nsub_; ++i) put_be(b, (int32_t)mask[r * nsub_ + i]);
      for (long i = 0; i < nsub_; ++i) put_be(b, crit ? crit[r * nsub_ + i] : 0.0f);
    });
  }

  // upper triangle of [npix][nmap][nmap] (write_matrix, output.f90:1031-1175)
  void matrix(const std::string &f, const double *cc) {
    if (f.empty()) return;
    std::vector<Col> cols;
    std::vector<std::pair<int, int>> ij;
    for (int i = 0; i < nmap_; ++i)
      for (int j = i; j < nmap_; ++j) {
        cols.push_back({"cc(" + std::to_string(i + 1) + "," + std::to_string(j + 1) + ")",
                        std::to_string(nsub_) + "D", "", (int)(8 * nsub_)});
        ij.push_back({i, j});
      }
    auto keys = [&](Header &h) {
      h.str("OBJTYPE", "madam.matrix", "Object type");
      healpix(h);
    };
    write_table(f, cols, nsm_, keys, [&](long long r, std::vector<unsigned char> &b) {
      for (auto e : ij)
        for (long q = 0; q < nsub_; ++q) {
          const long px = r * nsub_ + q;
          put_be(b, cc[(size_t)px * nmap_ * nmap_ + e.second * nmap_ + e.first]);
        }
    });
  }

  // every element gamma(i, j) of [npix][nmap][nmap], row i column j
  // (write_leakmatrix, output.f90:1181-1323)
  void leak(const std::string &f, const double *g) {
    if (f.empty()) return;
    std::vector<Col> cols;
    for (int i = 0; i < nmap_; ++i)
      for (int j = 0; j < nmap_; ++j)
        cols.push_back({"gamma(" + std::to_string(i + 1) + "," + std::to_string(j + 1) + ")",
                        std::to_string(nsub_) + "D", "", (int)(8 * nsub_)});
    auto keys = [&](Header &h) {
      h.str("OBJTYPE", "madam.leakmatrix", "Object type");
      healpix(h);
    };
    write_table(f, cols, nsm_, keys, [&](long long r, std::vector<unsigned char> &b) {
      for (int e = 0; e < nmap_ * nmap_; ++e)
        for (long q = 0; q < nsub_; ++q) put_be(b, g[(size_t)(r * nsub_ + q) * nmap_ * nmap_ + e]);
    });
  }

 private:
  void healpix(Header &h) {
    h.str("PIXTYPE", "HEALPIX", "HEALPIX Pixelisation");
    h.str("ORDERING", "NESTED", "Pixel ordering scheme");
    h.integer("NSIDE", p_.nside_map, "Resolution parameter for HEALPIX");
    h.integer("FIRSTPIX", 0, "First pixel # (0 based)");
    h.integer("LASTPIX", 12LL * p_.nside_map * p_.nside_map - 1, "Last pixel # (0 based)");
    h.logical("POLAR", nmap_ != 1, "Polarisation included (True/False)");
    h.str("POLCCONV", "COSMO", "Coord. convention for polarisation (COSMO/IAU)");
    h.str("EXTNAME", "FULL SKY MAP");
    h.str("OBJECT", "FULLSKY");
    h.str("INDXSCHM", "IMPLICIT", "Indexing : IMPLICIT or EXPLICIT");
    h.integer("GRAIN", 0, "Grain of pixel indexing");
    h.str("CREATOR", "Madam", "Software creating FITS file");
    h.integer("NODET", ndet_, "Number of detectors");
    h.real("FSAMPLE", p_.fsample, "Sampling frequency (Hz)");
    h.integer("NSIDESUB", p_.nside_submap, "Submap resolution");
    h.integer("NSIDECR", p_.nside_cross, "Crossing point resolution");
  }
  const Params &p_;
  long nsub_, nsm_, ndet_;
  int nmap_;
};

// <path_output><file_root>[_<set>][_<survey>] (parameter_control.f90:48-63,
// smadam.F90:1112-1116); a leading '!' of the root is kept in front
std::string stem(const Params &p, const std::string &set, const std::string &survey) {
  std::string path = p.path_output;
  if (!path.empty() && path.back() != '/') path += '/';
  std::string f = p.file_root;
  if (!set.empty()) f += "_" + set;
  if (!survey.empty()) f += "_" + survey;
  if (!f.empty() && f[0] == '!') return "!" + path + f.substr(1);
  return path + f;
}

// add_subchunk_id (smadam.F90:1285-1314): "_sub<i>of<n>" before the last
// '.' (at the end when there is none); one digit each below 10 subchunks,
// two from 10
std::string subchunk_id(const std::string &f, int isub, int nsub) {
  if (f.empty() || isub == 0) return f;
  char tag[32];
  if (nsub < 10) std::snprintf(tag, sizeof tag, "_sub%1dof%1d", isub, nsub);
  else std::snprintf(tag, sizeof tag, "_sub%02dof%02d", isub, nsub);
  const size_t dot = f.rfind('.');
  if (dot == std::string::npos) return f + tag;
  return f.substr(0, dot) + tag + f.substr(dot);
}

}  // namespace

void write_products(const FitsInput &in) {
  const Params &p = *in.par;
  const std::string root = stem(p, p.detsets[0].name, p.surveys[0].name);
  auto nm = [&](const std::string &suffix) {
    return resolve(subchunk_id(root + suffix, in.isubchunk, in.nsubchunk));
  };
  Tables t(p, in.nosubpix_map, in.nosubmaps_tot, in.ndet, in.nmap);
  if (p.do_map && in.map) t.map(nm("_map.fits"), in.map, in.mask, "madam.map");
  if (p.do_binmap && in.binmap) t.map(nm("_bmap.fits"), in.binmap, in.mask, "madam.binmap");
  if (in.first_call && p.do_hits && in.hits) t.hits(nm("_hmap.fits"), in.hits);
  if (in.first_call && p.do_mask && in.mask) t.mask(nm("_mask.fits"), in.mask, in.crit);
  if (in.first_call && p.do_matrix && in.cc_raw) t.matrix(nm("_wcov_inv.fits"), in.cc_raw);
  if (in.first_call && p.do_wcov && in.cc_inv) t.matrix(nm("_wcov.fits"), in.cc_inv);
  if (in.first_call && p.do_leakmatrix) {
    // file_leakmatrix = <stem>_leakmatrix (parameter_control.f90:61), then
    // write_leakmatrix appends _<detector>.fits (output.f90:1199)
    const std::string base = subchunk_id(root + "_leakmatrix", in.isubchunk, in.nsubchunk);
    for (const auto &lk : in.leak) t.leak(resolve(base + "_" + lk.first + ".fits"), lk.second);
  }
}

// ---- reading: the input mask (read_inmask, read_data.f90:90-190)
namespace {
std::string card_value(const std::string &card) {
  std::string v = card.size() > 10 ? card.substr(10) : "";
  const size_t q = v.find('\'');
  if (q != std::string::npos) {
    const size_t e = v.find('\'', q + 1);
    std::string t = v.substr(q + 1, e == std::string::npos ? std::string::npos : e - q - 1);
    while (!t.empty() && t.back() == ' ') t.pop_back();
    return t;
  }
  const size_t sl = v.find('/');
  if (sl != std::string::npos) v = v.substr(0, sl);
  size_t a = v.find_first_not_of(' '), b = v.find_last_not_of(' ');
  return a == std::string::npos ? "" : v.substr(a, b - a + 1);
}

// one header: keyword -> value; the stream is left after its END block
std::vector<std::pair<std::string, std::string>> read_header(FILE *f) {
  std::vector<std::pair<std::string, std::string>> kv;
  char block[2880];
  for (;;) {
    if (std::fread(block, 1, 2880, f) != 2880) fail("truncated FITS header");
    for (int c = 0; c < 36; ++c) {
      const std::string card(block + 80 * c, 80);
      std::string key = card.substr(0, 8);
      while (!key.empty() && key.back() == ' ') key.pop_back();
      if (key == "END") return kv;
      if (card.size() > 9 && card[8] == '=') kv.push_back({key, card_value(card)});
    }
  }
}

std::string get(const std::vector<std::pair<std::string, std::string>> &kv, const std::string &k,
                const std::string &dflt = "") {
  for (auto &e : kv)
    if (e.first == k) return e.second;
  return dflt;
}
}  // namespace

std::vector<float> read_mask_column(const std::string &file, long &nside, std::string &ordering) {
  FILE *f = std::fopen(file.c_str(), "rb");
  if (!f) fail("cannot open " + file);
  std::vector<float> out;
  try {
    auto prim = read_header(f);
    long long psize = 0;
    const long naxis = std::stol(get(prim, "NAXIS", "0"));
    if (naxis > 0) {
      psize = std::llabs(std::stoll(get(prim, "BITPIX", "8"))) / 8;
      for (long i = 1; i <= naxis; ++i) psize *= std::stoll(get(prim, "NAXIS" + std::to_string(i)));
    }
    std::fseek(f, (long)((psize + 2879) / 2880 * 2880), SEEK_CUR);
    auto ext = read_header(f);
    if (get(ext, "XTENSION") != "BINTABLE") fail(file + ": no binary table");
    const long long rowb = std::stoll(get(ext, "NAXIS1")), nrow = std::stoll(get(ext, "NAXIS2"));
    const std::string tf = get(ext, "TFORM1");
    size_t i = 0;
    while (i < tf.size() && isdigit((unsigned char)tf[i])) ++i;
    const long rep = i ? std::stol(tf.substr(0, i)) : 1;
    const char t = i < tf.size() ? tf[i] : 'E';
    const int w = t == 'E' || t == 'J' ? 4 : t == 'D' || t == 'K' ? 8 : t == 'I' ? 2 : 1;
    ordering = get(ext, "ORDERING");
    nside = std::stol(get(ext, "NSIDE", "0"));
    std::vector<unsigned char> row((size_t)rowb);
    out.reserve((size_t)(nrow * rep));
    for (long long r = 0; r < nrow; ++r) {
      if (std::fread(row.data(), 1, row.size(), f) != row.size()) fail(file + ": truncated table");
      for (long k = 0; k < rep; ++k) {
        const unsigned char *p = row.data() + k * w;
        uint64_t u = 0;
        for (int b = 0; b < w; ++b) u = (u << 8) | p[b];
        double v;
        if (t == 'E') {
          uint32_t u32 = (uint32_t)u;
          float x;
          std::memcpy(&x, &u32, 4);
          v = x;
        } else if (t == 'D') {
          std::memcpy(&v, &u, 8);
        } else if (t == 'J') {
          v = (double)(int32_t)(uint32_t)u;
        } else if (t == 'K') {
          v = (double)(int64_t)u;
        } else if (t == 'I') {
          v = (double)(int16_t)(uint16_t)u;
        } else if (t == 'L') {
          v = p[0] == 'T' ? 1.0 : 0.0;
        } else {
          v = (double)p[0];
        }
        out.push_back((float)v);
      }
    }
  } catch (...) {
    std::fclose(f);
    throw;
  }
  std::fclose(f);
  return out;
}

void write_subset_products(const SubsetFits &in) {
  // run_subsets (smadam.F90:1112-1224): names from the set and survey; a
  // file that exists already is not written (skip_existing there)
  const Params &p = *in.par;
  const std::string sub = stem(p, in.set, in.survey);
  auto fresh = [&](const std::string &f0) {
    const std::string f = subchunk_id(f0, in.isubchunk, in.nsubchunk);
    if (!f.empty() && f[0] == '!') return f.substr(1);  // overwrite, as cfitsio does
    return exists(f) ? std::string() : f;
  };
  Tables t(p, in.nosubpix_map, in.nosubmaps_tot, in.ndet, in.nmap);
  const bool last_map = in.pass == in.npass && p.do_map;
  if (last_map) t.map(fresh(sub + "_map.fits"), in.binmap, in.mask, "madam.binmap");
  else if (p.do_binmap || p.do_map) t.map(fresh(sub + "_bmap.fits"), in.binmap, in.mask, "madam.binmap");
  if (in.pass != 1) return;
  if (p.do_hits) t.hits(fresh(sub + "_hmap.fits"), in.hits);
  if (p.do_matrix) t.matrix(fresh(sub + "_wcov_inv.fits"), in.cc_raw);
  const std::string lbase = subchunk_id(sub + "_leakmatrix.fits", in.isubchunk, in.nsubchunk);
  if (p.do_leakmatrix && !exists(lbase))
    for (const auto &lk : in.leak) t.leak(resolve(lbase + "_" + lk.first + ".fits"), lk.second);
  if (p.do_wcov) t.matrix(fresh(sub + "_wcov.fits"), in.cc_inv);
  if (p.do_mask) t.mask(fresh(sub + "_mask.fits"), in.mask, in.crit);
}

}  // namespace madam
