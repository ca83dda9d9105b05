// Host-side configuration of one destripe() call: the parstring parser, the
// default values, the detector / PSD table and the derived layout.
//
// Mirrors the reference's configuration layer:
//   defaults          commonparam.f90:200-305 (set_parameter_defaults)
//   parstring parser  inputparam.f90:24-67 (read_parameters), 169-371
//                     (read_line), 375-492 (detset / survey), 498-505
//   detector table    inputparam.f90:73-163 (read_detectors)
//   derived values    parameter_control.f90:27-409 (init_parameters)
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace madam {

// Error raised wherever the reference calls abort_mpi / stop.  The C-ABI
// converts it to a status code and a message; the caller's process survives.
struct Error : std::runtime_error {
  explicit Error(const std::string &m) : std::runtime_error(m) {}
};
[[noreturn]] inline void fail(const std::string &m) { throw Error(m); }

// A Fortran default-real literal (single precision) widened to double; the
// reference's thresholds and defaults such as 1e-12 or 1e-30 are written this
// way, so the exact double values differ from the decimal ones.
#ifdef __CUDACC__
#define MADAM_FSP_QUAL __host__ __device__
#else
#define MADAM_FSP_QUAL
#endif
MADAM_FSP_QUAL inline constexpr double fsp(float x) { return (double)x; }

struct Params {
  double fsample = 1;
  bool concatenate_messages = true, allreduce = false, reassign_submaps = true;
  bool noise_weights_from_psd = false, radiometers = true;
  long psd_downsample = 10, psdlen = 1000000;
  long nsubchunk = 0, isubchunk = 0;
  bool checknan = false;
  double diagfilter = 0;
  bool sync_output = true, skip_existing = false, write_cut = false;
  bool binary_output = false;
  long nwrite_binary = 10;
  int basis_func = 4;
  long basis_order = 0;
  bool bin_subsets = false, mcmode = false;
  double good_baseline_fraction = 0;
  bool incomplete_matrices = false;
  long info = 2;
  long nside_map = 512, nside_cross = -1, nside_submap = 16;
  double time_unit = -5;
  long pixmode_map = 2, pixmode_cross = 2;
  double pixlim_map = fsp(1e-6f), pixlim_cross = fsp(1e-3f);
  bool allow_decoupling = false;
  double dnshort = -1;
  bool kfirst = true, kfilter = false, unaligned_fft = false;
  double cglimit = fsp(1e-12f);
  long iter_min = 3, iter_max = 1000;
  long precond_width_min = 10, precond_width_max = 100;
  bool use_fprecond = false, use_cgprecond = false;
  long mode_detweight = 0;
  bool rm_monopole = false, temperature_only = false;
  bool flag_by_horn = false, force_pol = false;
  std::string file_inmask, file_spectrum, file_gap, file_root = "madam",
      path_output, unit_tod = "unknown", file_gap_out, file_mc, file_covmat;
  bool write_tod = false;
  bool do_map = true, do_binmap = false, do_hits = false, do_mask = false,
       do_matrix = false, do_wcov = false, do_base = false,
       do_leakmatrix = false;
  long nthreads = 1;
  int ndetset = 0, nsurvey = 0;
  // detector sets and surveys (inputparam.f90:375-492); entry 0 is the full
  // set / span, whose name an "all" definition sets
  struct DetSet {
    std::string name;
    std::vector<std::string> dets;
    bool nopol = false;
  };
  struct Survey {
    std::string name;
    std::vector<double> starts, stops;
  };
  std::vector<DetSet> detsets = std::vector<DetSet>(1);
  std::vector<Survey> surveys = std::vector<Survey>(1);
};

// Parse "key = value;key = value;..." exactly as read_parameters does,
// including dnshort = nint(base_first * fsample) and the 1e10 default.
Params parse_parstring(const char *parstring);

struct Detector {
  std::string name;
  int npsd = 1;
  bool has_psd = false;
  std::vector<double> psdstarts, sigmas, weights, plateaus;
  std::vector<double> psdfreqs;            // shared bins
  std::vector<std::vector<double>> psds;   // [ipsd][bin]
};

std::vector<Detector> read_detectors(const Params &p, const char *detstring,
                                     long ndet, const double *detweights,
                                     const long *npsd, long npsdtot,
                                     const double *psdstarts, long npsdbin,
                                     const double *psdfreqs, long npsdval,
                                     const double *psdvals);

// interpolate_psd (noise_routines.f90:130-190): log-log interpolation with a
// monotone bracket walk (targets are expected in ascending order).
void interpolate_psd(const std::vector<double> &freq,
                     const std::vector<double> &psd, const double *target,
                     double *out, long nout);

// The noise spectra of file_spectrum (read_spectrum, noise_routines.f90:
// 505-596): the log frequencies of the table, and per detector (in the
// detectors' order) the log spectrum of its column and its sigma.  Columns
// are matched to detectors as the reference matches them: the first column
// whose name contains the detector's name.
struct SpectrumFile {
  std::vector<double> logf;
  std::vector<std::vector<double>> logspec;
  std::vector<double> sigma;
};
SpectrumFile read_spectrum_file(const std::string &path, const std::vector<Detector> &dets);

// get_spectrum_file (noise_routines.f90:600-634): the spectrum of one
// detector at ascending frequencies f (log-log interpolation with the
// reference's monotone bracket walk and its clamp to the table's ends).
void spectrum_from_file(const SpectrumFile &sf, int idet, const double *f, double *out,
                        long nout);

// psd_index_det (noise_routines.f90:211-236); 0-based, -1 if none.
int psd_index_det(const Detector &d, double t);

}  // namespace madam
