// Test harness of the FITS writer (libmadam_b200/csrc/fits.cpp): writes the
// products of a made-up nside 4 run with known values, so that the files can
// be checked on a machine without a GPU.  Built and run by
// tests/test_fits_writer.py:  fits_harness <output dir> <nmap> [<file_root>]
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <string>
#include <vector>

#include "fits.h"
#include "params.h"

int main(int argc, char **argv) {
  if (argc != 3 && argc != 4) return 2;
  const std::string dir = argv[1];
  const int nmap = std::atoi(argv[2]);
  try {
    const std::string root = argc == 4 ? argv[3] : "run";
    const std::string pars = "nside_map = 4; nside_submap = 2; file_root = " + root +
                             "; path_output = " + dir +
                             "; write_map = T; write_binmap = T; write_hits = T; " +
                             "write_mask = T; write_matrix = T; write_wcov = T; " +
                             "write_leakmatrix = T; unit_tod = K_CMB;";
    madam::Params p = madam::parse_parstring(pars.c_str());
    const long nsub = 4, nsm = 48, npix = nsub * nsm, nn = (long)nmap * nmap;
    std::vector<double> map(npix * nmap), binmap(npix * nmap), cc_raw(npix * nn),
        cc_inv(npix * nn), leak(npix * nn);
    std::vector<int> hits(npix), mask(npix);
    std::vector<float> crit(npix);
    for (long px = 0; px < npix; ++px) {
      for (int j = 0; j < nmap; ++j) {
        map[px * nmap + j] = px + 0.25 * j;
        binmap[px * nmap + j] = -(px + 0.5 * j);
      }
      for (long e = 0; e < nn; ++e) {
        cc_raw[px * nn + e] = px + e / 16.0;
        cc_inv[px * nn + e] = 1.0 / (1 + px + e);
        leak[px * nn + e] = px * 100.0 + e;
      }
      hits[px] = (int)(3 * px);
      mask[px] = px % 5 != 0;
      crit[px] = 0.5f * px;
    }
    madam::FitsInput in;
    in.par = &p;
    in.nosubpix_map = nsub;
    in.nosubmaps_tot = nsm;
    in.ndet = 1;
    in.nmap = nmap;
    in.map = map.data();
    in.binmap = binmap.data();
    in.hits = hits.data();
    in.mask = mask.data();
    in.crit = crit.data();
    in.cc_raw = cc_raw.data();
    in.cc_inv = cc_inv.data();
    in.leak.push_back({"d0", leak.data()});
    madam::write_products(in);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
