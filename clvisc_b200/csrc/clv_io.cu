// Host-side writer of the reference's text tables (hypersf.dat, sf_txyz.dat,
// pimnsf.dat: numpy.savetxt with fmt='%.6e' and a header, ideal.py:304-312,
// visc.py:413-419). The rows are formatted in parallel host threads and
// written in order; the bytes equal numpy.savetxt's: '# ' + header + '\n',
// then each row's values as %.6e of the value as a double, separated by one
// space, ending in '\n'. Python prints every NaN as 'nan' (C's printf writes
// '-nan' for a NaN with the sign bit set), which this writer follows.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/clvisc_b200.h"

namespace clv_host {
int set_error(int code, const std::string& msg);
}

namespace {

inline int format_value(char* out, double v) {
  if (std::isnan(v)) {
    std::memcpy(out, "nan", 3);
    return 3;
  }
  return std::snprintf(out, 32, "%.6e", v);
}

template <class real> void format_rows(const real* data, long long r0, long long r1, int cols, std::string* out) {
  char buf[40];
  out->clear();
  out->reserve((size_t)(r1 - r0) * cols * 14);
  for (long long r = r0; r < r1; r++) {
    for (int c = 0; c < cols; c++) {
      const int n = format_value(buf, (double)data[r * cols + c]);
      out->append(buf, (size_t)n);
      out->push_back(c + 1 < cols ? ' ' : '\n');
    }
  }
}

}  // namespace

extern "C" {

int clv_write_table(const char* path, const char* header, const void* data, int precision, long long rows, int cols) {
  if (!path || (rows > 0 && !data) || rows < 0 || cols < 1 || (precision != 4 && precision != 8))
    return clv_host::set_error(CLV_ERR_INVALID, "write_table: bad argument");
  FILE* f = std::fopen(path, "wb");
  if (!f) return clv_host::set_error(CLV_ERR_INVALID, std::string("write_table: cannot open ") + path);
  int rc = CLV_OK;
  if (header) {
    const std::string h = std::string("# ") + header + "\n";
    if (std::fwrite(h.data(), 1, h.size(), f) != h.size()) rc = CLV_ERR_INVALID;
  }
  // rows in blocks, formatted by up to 16 threads, written in order
  const long long block = 1 << 16;
  unsigned hw = std::thread::hardware_concurrency();
  const int nt = (int)std::max(1u, std::min(16u, hw ? hw : 1u));
  std::vector<std::string> bufs(nt);
  for (long long base = 0; base < rows && rc == CLV_OK; base += block * nt) {
    std::vector<std::thread> th;
    for (int t = 0; t < nt; t++) {
      const long long r0 = base + t * block, r1 = std::min(rows, r0 + block);
      if (r0 >= r1) {
        bufs[t].clear();
        continue;
      }
      if (precision == 4)
        th.emplace_back(format_rows<float>, (const float*)data, r0, r1, cols, &bufs[t]);
      else
        th.emplace_back(format_rows<double>, (const double*)data, r0, r1, cols, &bufs[t]);
    }
    for (auto& x : th) x.join();
    for (int t = 0; t < nt && rc == CLV_OK; t++)
      if (!bufs[t].empty() && std::fwrite(bufs[t].data(), 1, bufs[t].size(), f) != bufs[t].size())
        rc = CLV_ERR_INVALID;
  }
  if (std::fclose(f) != 0) rc = CLV_ERR_INVALID;
  if (rc != CLV_OK) return clv_host::set_error(rc, std::string("write_table: write failed: ") + path);
  return CLV_OK;
}

}  // extern "C"
