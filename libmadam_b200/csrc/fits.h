// FITS products of destripe() (fits.cpp).
#pragma once

#include <string>
#include <utility>
#include <vector>

#include "params.h"

namespace madam {

// Full-sky host arrays at nside_map; null pointers skip the product.
struct FitsInput {
  const Params *par = nullptr;
  long nosubpix_map = 0, nosubmaps_tot = 0, ndet = 0;
  int nmap = 0;
  bool first_call = true;          // destripe (all products) or destripe_with_cache (maps)
  int isubchunk = 0, nsubchunk = 0;  // subchunk pass: names get _sub<i>of<n>
  const double *map = nullptr;     // [npix][nmap]
  const double *binmap = nullptr;  // [npix][nmap]
  const int *hits = nullptr;       // [npix]
  const int *mask = nullptr;       // [npix]
  const float *crit = nullptr;     // [npix]
  const double *cc_raw = nullptr;  // [npix][nmap][nmap] before inversion
  const double *cc_inv = nullptr;  // [npix][nmap][nmap] after inversion
  // leakage matrices [npix][nmap][nmap] (row i, column j) by detector name
  std::vector<std::pair<std::string, const double *>> leak;
};

void write_products(const FitsInput &in);

// One subset of run_subsets: the products of one (pass, detector set, survey).
struct SubsetFits {
  const Params *par = nullptr;
  long nosubpix_map = 0, nosubmaps_tot = 0, ndet = 0;
  int nmap = 0, pass = 1, npass = 1;
  int isubchunk = 0, nsubchunk = 0;
  std::string set, survey;
  const double *binmap = nullptr;
  const int *hits = nullptr, *mask = nullptr;
  const float *crit = nullptr;
  const double *cc_raw = nullptr, *cc_inv = nullptr;
  std::vector<std::pair<std::string, const double *>> leak;
};

void write_subset_products(const SubsetFits &in);

// The first column of the first binary table of a FITS file (the input mask
// of read_inmask, read_data.f90:90-190) with its NSIDE and ORDERING keys.
std::vector<float> read_mask_column(const std::string &file, long &nside, std::string &ordering);

}  // namespace madam
