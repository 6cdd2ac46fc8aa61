// Output files of the LCS diagnostics: the reference's write_lcs / write_ftle layout
// (src/io_nohdf5_m.f90:47-133, 183-264, 266-332): a Tecplot ASCII file per FTLE frame,
// ./cfd2lcs_output/<label>_<index>.dat, with a text header and one BLOCK of values per
// variable, ten ES14.6 values per line.
//
// The frame's device fields are copied into pinned staging memory by cudaMemcpyAsync on the
// engine's stream; a worker thread waits for the copies' event, formats the blocks (several
// threads per block) and writes the file, so the GPU goes on with the next updates meanwhile.
// At most two frames are staged at once; a third waits for a staging buffer.
#pragma once

#include <cuda_runtime.h>

#include <condition_variable>
#include <cstdint>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace cfd2lcs {

// Fortran ESw.d editing of v in exactly w characters (right-justified; E+dd exponent, or +ddd
// without the E when it has three digits; NaN / Infinity spelled as gfortran does).
void format_es(double v, int w, int d, char *out);

// File name index of write_lcs (src/io_nohdf5_m.f90:72-118): the decimal index, except that
// 1000..9999 are zero-padded to ten digits (the reference's i10.10 for that range).  False
// outside -999999999..999999999.
bool lcs_file_index(long long findex, std::string &out);

struct OutputBlock {
  enum Kind { STAGED_F64, STAGED_F32, LINE_X, LINE_Y, LINE_Z, FLAG, ZERO } kind = ZERO;
  size_t offset = 0;  // byte offset of a staged block in the staging buffer
};

struct OutputJob {
  std::string path;
  std::string header;
  std::vector<OutputBlock> blocks;
  long n[3] = {0, 0, 0};
  // grid lines (x by i, y by j, z by k) and interior flags, shared with the engine
  std::shared_ptr<const std::vector<double>> lines[3];
  // non-rectilinear grids: the node coordinates themselves (interior, i fastest), used instead
  // of the lines
  std::shared_ptr<const std::vector<double>> coords[3];
  std::shared_ptr<const std::vector<int8_t>> flags;
  long points = -1;  // >= 0: POINT packing of that many particles (blocks x, y, z), one per line
  cudaEvent_t ready = nullptr;  // staged copies complete
  int buffer = -1;
};

class LcsWriter {
 public:
  LcsWriter();
  ~LcsWriter();
  // A pinned staging buffer of at least `bytes` (waits while both are in use); its index.
  int acquire(size_t bytes, void **ptr, std::string &msg);
  // Queues a job whose staged copies were enqueued before job.ready was recorded.
  void submit(OutputJob &&job);
  // Waits until every queued file is written.
  void flush();
  // First error of a finished job (empty if none); cleared by the call.
  std::string take_error();

 private:
  void run();
  bool write_job(const OutputJob &job, const char *staging, std::string &err);

  struct Buf {
    void *ptr = nullptr;
    size_t bytes = 0;
    bool busy = false;
  };
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<OutputJob> queue_;
  Buf bufs_[2];
  bool stop_ = false;
  int active_ = 0;
  std::string error_;
  std::thread worker_;
};

}  // namespace cfd2lcs
