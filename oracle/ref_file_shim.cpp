/*
 * C-ABI shim around the reference's table loader (TEST INFRASTRUCTURE ONLY).
 *
 * Compiled by oracle/build.py from input/File.h and time/Time.h where they lie into
 * oracle/_ref/libref_file.so.  Nothing from the reference is copied here: this file
 * instantiates File<float> and calls its public count and load, so tests can pin the
 * CSV restatement (oracle/csv_oracle.py) against the real code and the benchmark can
 * time the reference's fscanf path.  Only load and count are used, so the generator
 * that input/File.h declares (randdataset.c) is never needed.
 */
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>

#include "input/File.h"

namespace {
struct Quiet {  // File<T>::load prints progress lines
  std::streambuf *old;
  std::ostringstream sink;
  Quiet() : old(std::cout.rdbuf(sink.rdbuf())) {}
  ~Quiet() { std::cout.rdbuf(old); }
};
}  // namespace

extern "C" {

/* File<float>(fname, gpu=false) counts the file (input/File.h:108-132). */
void ref_file_count(const char *path, uint64_t *n, uint64_t *d) {
  File<float> f(std::string(path), false);
  *n = f.rows();
  *d = f.items();
}

/* File<float>(fname, false, n, d) with set_transpose(true), load(data): the n x d table
 * column-major into out (n * d floats). */
void ref_file_load(const char *path, uint64_t n, uint64_t d, float *out) {
  File<float> f(std::string(path), false, n, d);
  f.set_transpose(true);
  float *data = nullptr;
  {
    Quiet q;
    f.load(data);
  }
  std::memcpy(out, data, sizeof(float) * n * d);
  std::free(data);
}

}  // extern "C"
