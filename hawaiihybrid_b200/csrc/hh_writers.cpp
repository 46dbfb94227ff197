// CF and SF text writers (write_correlation_function_ext / write_spectral_function_ext,
// src/hawaii.c:4150-4284) with the same bytes as the reference's fprintf loop: the
// header, then one "%.2f %.10e\n" (CF) or "%.10f   %.10e\n" (SF) line per point.  The
// lines are formatted by snprintf in parallel chunks, one per host thread, into
// memory and written with one fwrite, instead of one fprintf per line.
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "../../include/hh_cuda.h"

namespace {

// formats lines [b, e) into out
template <typename Fmt> void format_chunk(size_t b, size_t e, Fmt fmt, std::string *out) {
  char line[128];
  out->clear();
  out->reserve((e - b) * 32);
  for (size_t i = b; i < e; ++i) {
    const int k = fmt(line, sizeof line, i);
    if (k > 0) out->append(line, (size_t)std::min<int>(k, (int)sizeof line - 1));
  }
}

template <typename Fmt>
long write_table(FILE *fp, const char *len_key, double T, double ntraj, size_t len, Fmt fmt) {
  if (!fp) return HH_E_INVALID_ARGUMENT;
  const int fd = fileno(fp);
  if (ftruncate(fd, 0) < 0) return HH_E_INVALID_ARGUMENT;
  rewind(fp);
  time_t raw;
  time(&raw);
  struct tm tmv;
  localtime_r(&raw, &tmv);
  char hdr[512];
  const int nh = snprintf(hdr, sizeof hdr,
                          "# HAWAII HYBRID v0.1\n# Saved on %04d-%02d-%02d %02d:%02d:%02d\n# TEMPERATURE: %.2f\n"
                          "# AVERAGE OVER %.2f TRAJECTORIES\n# %s: %zu\n",
                          tmv.tm_year + 1900, tmv.tm_mon + 1, tmv.tm_mday, tmv.tm_hour, tmv.tm_min, tmv.tm_sec, T,
                          ntraj, len_key, len);
  unsigned nt = std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
  if (len < 4096) nt = 1;
  std::vector<std::string> parts(nt);
  std::vector<std::thread> th;
  for (unsigned w = 0; w < nt; ++w) {
    const size_t b = len * w / nt, e = len * (w + 1) / nt;
    if (nt == 1) format_chunk(b, e, fmt, &parts[w]);
    else th.emplace_back(format_chunk<Fmt>, b, e, fmt, &parts[w]);
  }
  for (auto &t : th) t.join();
  long n = 0;
  if (fwrite(hdr, 1, (size_t)nh, fp) != (size_t)nh) return HH_E_INVALID_ARGUMENT;
  n += nh;
  for (const auto &p : parts) {
    if (!p.empty() && fwrite(p.data(), 1, p.size(), fp) != p.size()) return HH_E_INVALID_ARGUMENT;
    n += (long)p.size();
  }
  if (fflush(fp) != 0) return HH_E_INVALID_ARGUMENT;
  if (fsync(fd) < 0) return HH_E_INVALID_ARGUMENT;
  return n;
}

}  // namespace

extern "C" {

long hh_write_correlation_function_ext(FILE *fp, const double *t, const double *data, size_t len,
                                       double Temperature, double ntraj, int normalized) {
  if (!t || !data) return HH_E_INVALID_ARGUMENT;
  if (!normalized && !(ntraj > 0)) return HH_E_INVALID_ARGUMENT;
  const double s = normalized ? 1.0 : ntraj;
  return write_table(fp, "MAXIMUM TRAJECTORY LENGTH", Temperature, ntraj, len,
                     [=](char *b, size_t n, size_t i) {
                       return snprintf(b, n, "%.2f %.10e\n", t[i], normalized ? data[i] : data[i] / s);
                     });
}

long hh_write_spectral_function_ext(FILE *fp, const double *nu, const double *data, size_t len,
                                    double Temperature, double ntraj, int normalized) {
  if (!nu || !data) return HH_E_INVALID_ARGUMENT;
  if (!normalized && !(ntraj > 0)) return HH_E_INVALID_ARGUMENT;
  const double s = normalized ? 1.0 : ntraj;
  return write_table(fp, "SPECTRAL FUNCTION LENGTH", Temperature, ntraj, len,
                     [=](char *b, size_t n, size_t i) {
                       return snprintf(b, n, "%.10f   %.10e\n", nu[i], normalized ? data[i] : data[i] / s);
                     });
}

}  // extern "C"
