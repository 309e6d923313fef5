// spectrum.h - emission spectra and their inverse CDF (js/spectra.js).
//
// The reference's host builds the wavelength-sampling table with Spectrum.inverseCDF
// (js/spectra.js:28-61) over 390..750 nm with 1024 spectrum samples and 4*1024 ICDF entries,
// storing into Float32Arrays (each store rounds to float) while the arithmetic runs in double.
// This restatement keeps both: double arithmetic, float storage.
#pragma once
#include <algorithm>
#include <cmath>
#include <vector>

#include "snelly.h"

namespace snelly {

inline double spectrum_value(const snelly_spectrum& s, double wavelength_nm) {
  if (s.kind == SNELLY_SPECTRUM_FLAT) {  // js/spectra.js:123-128
    if (wavelength_nm < s.band_min) return 0.0;
    if (wavelength_nm > s.band_max) return 0.0;
    return 1.0;
  }
  // BlackbodySpectrum.spectrum, js/spectra.js:179-184 (wavelength relative to 360 nm)
  double b = 1.43877737467e7 / (wavelength_nm * (double)s.temperature);
  double l = wavelength_nm / 360.0;
  return 1.0 / (l * l * l * l * l * (std::exp(b) - 1.0));
}

inline std::vector<float> inverse_cdf(const snelly_spectrum& s, double lmin = 390.0, double lmax = 750.0,
                                      int nsamples = 1024) {
  std::vector<float> icdf(4 * nsamples);
  if (s.kind == SNELLY_SPECTRUM_MONO) {  // js/spectra.js:76-86
    double w = std::max(lmin, std::min((double)s.wavelength, lmax));
    float off = (float)((w - lmin) / (lmax - lmin));
    std::fill(icdf.begin(), icdf.end(), off);
    return icdf;
  }
  std::vector<float> cdf(nsamples + 1);
  double dl = (lmax - lmin) / nsamples;
  cdf[0] = 0.0f;
  for (int n = 0; n < nsamples; ++n) cdf[n + 1] = (float)((double)cdf[n] + spectrum_value(s, lmin + dl * n));
  double sum = cdf[nsamples];
  for (int n = 0; n < nsamples; ++n) cdf[n + 1] = (float)((double)cdf[n + 1] / sum);
  cdf[nsamples] = 1.0f;
  int idx = 0;
  for (int n = 0; n < 4 * nsamples; ++n) {
    double xi = std::min((double)(n + 1) / (4.0 * nsamples), 1.0);
    while ((double)cdf[idx] < xi) idx++;
    idx = std::max(1, idx);
    double lo = cdf[idx - 1], hi = cdf[idx];
    double ilo = (idx - 1.0) / nsamples;
    icdf[n] = (float)(ilo + (1.0 / nsamples) * (xi - lo) / (hi - lo));
  }
  return icdf;
}

}  // namespace snelly
