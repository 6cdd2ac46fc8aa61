// Tecplot ASCII output of the FTLE frames (write_ftle, src/io_nohdf5_m.f90:183-264, and
// write_data_from_master :266-332 at one rank).
#include "writer.h"

#include <sys/stat.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>

namespace cfd2lcs {

void format_es(double v, int w, int d, char *out) {
  char buf[64];
  int len;
  if (std::isnan(v)) {
    len = std::snprintf(buf, sizeof(buf), "NaN");
  } else if (std::isinf(v)) {
    len = std::snprintf(buf, sizeof(buf), "%s", v < 0 ? "-Infinity" : "Infinity");
  } else {
    // one digit before the point, d after, correctly rounded: d.ddddddE+xx
    len = std::snprintf(buf, sizeof(buf), "%.*E", d, v);
    char *e = std::strchr(buf, 'E');
    if (e && len - (int)(e - buf) - 2 == 3) {  // three exponent digits: +ddd, the E dropped
      std::memmove(e, e + 1, (size_t)(len - (e - buf)));
      len--;
    }
  }
  if (len > w) {  // does not fit: asterisks, as Fortran editing does
    std::memset(out, '*', (size_t)w);
    return;
  }
  std::memset(out, ' ', (size_t)(w - len));
  std::memcpy(out + (w - len), buf, (size_t)len);
}

bool lcs_file_index(long long f, std::string &out) {
  if (f < -999999999LL || f > 999999999LL) return false;
  char buf[32];
  if (f >= 1000 && f <= 9999) std::snprintf(buf, sizeof(buf), "%010lld", f);
  else std::snprintf(buf, sizeof(buf), "%lld", f);
  out = buf;
  return true;
}

LcsWriter::LcsWriter() { worker_ = std::thread([this] { run(); }); }

LcsWriter::~LcsWriter() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  cv_.notify_all();
  if (worker_.joinable()) worker_.join();
  for (Buf &b : bufs_)
    if (b.ptr) cudaFreeHost(b.ptr);
}

int LcsWriter::acquire(size_t bytes, void **ptr, std::string &msg) {
  std::unique_lock<std::mutex> lk(mu_);
  cv_.wait(lk, [&] { return !bufs_[0].busy || !bufs_[1].busy; });
  const int i = !bufs_[0].busy ? 0 : 1;
  Buf &b = bufs_[i];
  if (b.bytes < bytes) {
    if (b.ptr) cudaFreeHost(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
    cudaError_t e = cudaMallocHost(&b.ptr, std::max<size_t>(bytes, 1));
    if (e != cudaSuccess) {
      b.ptr = nullptr;
      msg = std::string("write_lcs: pinned staging allocation failed: ") + cudaGetErrorString(e);
      return -1;
    }
    b.bytes = bytes;
  }
  b.busy = true;
  *ptr = b.ptr;
  return i;
}

void LcsWriter::submit(OutputJob &&job) {
  {
    std::lock_guard<std::mutex> lk(mu_);
    queue_.push_back(std::move(job));
  }
  cv_.notify_all();
}

void LcsWriter::flush() {
  std::unique_lock<std::mutex> lk(mu_);
  cv_.wait(lk, [&] { return queue_.empty() && active_ == 0; });
}

std::string LcsWriter::take_error() {
  std::lock_guard<std::mutex> lk(mu_);
  std::string e;
  e.swap(error_);
  return e;
}

void LcsWriter::run() {
  for (;;) {
    OutputJob job;
    const char *staging = nullptr;
    {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait(lk, [&] { return stop_ || !queue_.empty(); });
      if (queue_.empty()) return;  // stop requested and nothing left
      job = std::move(queue_.front());
      queue_.pop_front();
      active_++;
      if (job.buffer >= 0) staging = static_cast<const char *>(bufs_[job.buffer].ptr);
    }
    std::string err;
    if (job.ready) {
      const cudaError_t e = cudaEventSynchronize(job.ready);
      if (e != cudaSuccess) err = std::string("write_lcs: staging copy failed: ") + cudaGetErrorString(e);
      cudaEventDestroy(job.ready);
    }
    if (err.empty()) write_job(job, staging, err);
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (job.buffer >= 0) bufs_[job.buffer].busy = false;
      active_--;
      if (!err.empty() && error_.empty()) error_ = err;
    }
    cv_.notify_all();
  }
}

namespace {

constexpr int kPerLine = 10;  // NDATA_PER_LINE, src/io_nohdf5_m.f90:40
constexpr int kWidth = 14, kDigits = 6;  // ASCII_FMT = 'ES14.6', :41

// formats values [a, b) of a block (a a multiple of ten) into text, ten per line
template <typename Get>
void format_range(long a, long b, long count, const Get &get, std::string &s) {
  s.clear();
  const long nl = (b - a + kPerLine - 1) / kPerLine;
  s.reserve((size_t)((b - a) * kWidth + nl));
  char cell[kWidth];
  for (long q = a; q < b; q++) {
    format_es(get(q), kWidth, kDigits, cell);
    s.append(cell, kWidth);
    if ((q + 1) % kPerLine == 0 || q + 1 == count) s.push_back('\n');
  }
}

bool mkdir_p(const std::string &dir) {
  struct stat st;
  if (stat(dir.c_str(), &st) == 0) return S_ISDIR(st.st_mode);
  return mkdir(dir.c_str(), 0755) == 0 || errno == EEXIST;
}

}  // namespace

bool LcsWriter::write_job(const OutputJob &job, const char *staging, std::string &err) {
  const std::string dir = job.path.substr(0, job.path.find_last_of('/'));
  if (!dir.empty() && !mkdir_p(dir)) {
    err = "write_lcs: cannot create " + dir;
    return false;
  }
  FILE *fp = std::fopen(job.path.c_str(), "w");
  if (!fp) {
    err = "write_lcs: cannot open " + job.path;
    return false;
  }
  std::setvbuf(fp, nullptr, _IOFBF, 1 << 22);
  bool ok = std::fwrite(job.header.data(), 1, job.header.size(), fp) == job.header.size();
  if (job.points >= 0) {
    // write_tracers: '(3ES14.6)' per particle
    std::string out;
    out.reserve((size_t)job.points * (3 * kWidth + 1));
    char cell[kWidth];
    for (long q = 0; q < job.points && ok; q++) {
      for (int c = 0; c < 3; c++) {
        const OutputBlock &b = job.blocks[c];
        const double v = b.kind == OutputBlock::STAGED_F64 ? reinterpret_cast<const double *>(staging + b.offset)[q]
                                                           : (double)reinterpret_cast<const float *>(staging + b.offset)[q];
        format_es(v, kWidth, kDigits, cell);
        out.append(cell, kWidth);
      }
      out.push_back('\n');
    }
    if (ok && !out.empty()) ok = std::fwrite(out.data(), 1, out.size(), fp) == out.size();
    if (std::fclose(fp) != 0) ok = false;
    if (!ok) err = "write_lcs: write failed for " + job.path;
    return ok;
  }
  const long ni = job.n[0], nj = job.n[1], nk = job.n[2];
  const long count = ni * nj * nk;
  const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  const long nthreads = std::max(1L, std::min<long>(hw, count / 4096));
  std::vector<std::string> parts((size_t)nthreads);
  for (const OutputBlock &b : job.blocks) {
    if (!ok) break;
    const double *f64 = staging ? reinterpret_cast<const double *>(staging + b.offset) : nullptr;
    const float *f32 = staging ? reinterpret_cast<const float *>(staging + b.offset) : nullptr;
    const double *lx = job.lines[0] ? job.lines[0]->data() : nullptr;
    const double *ly = job.lines[1] ? job.lines[1]->data() : nullptr;
    const double *lz = job.lines[2] ? job.lines[2]->data() : nullptr;
    const int8_t *fl = job.flags ? job.flags->data() : nullptr;
    const double *cx = job.coords[0] ? job.coords[0]->data() : nullptr;
    const double *cy = job.coords[1] ? job.coords[1]->data() : nullptr;
    const double *cz = job.coords[2] ? job.coords[2]->data() : nullptr;
    auto get = [&](long q) -> double {
      switch (b.kind) {
        case OutputBlock::STAGED_F64: return f64[q];
        case OutputBlock::STAGED_F32: return (double)f32[q];
        case OutputBlock::LINE_X: return cx ? cx[q] : lx[q % ni];
        case OutputBlock::LINE_Y: return cy ? cy[q] : ly[(q / ni) % nj];
        case OutputBlock::LINE_Z: return cz ? cz[q] : lz[q / (ni * nj)];
        case OutputBlock::FLAG: return fl ? (double)fl[q] : 0.0;
        default: return 0.0;
      }
    };
    // line-aligned ranges, one per thread
    const long per = ((count / nthreads + kPerLine - 1) / kPerLine) * kPerLine;
    std::vector<std::thread> th;
    for (long t = 0; t < nthreads; t++) {
      const long a = std::min(count, t * per), e = std::min(count, (t + 1) * per);
      th.emplace_back([&, a, e, t] { format_range(a, e, count, get, parts[(size_t)t]); });
    }
    for (auto &x : th) x.join();
    for (const std::string &s : parts)
      if (ok && !s.empty()) ok = std::fwrite(s.data(), 1, s.size(), fp) == s.size();
  }
  if (std::fclose(fp) != 0) ok = false;
  if (!ok) err = "write_lcs: write failed for " + job.path;
  return ok;
}

}  // namespace cfd2lcs
