// Table files: the reference's comma-separated text read on the device, and a binary
// column-major format.
//
// The reference loads a table with File<float>::load (input/File.h:233-265, 306-330):
// fscanf("%f,%f,...,%f") once per object line, transposed into column-major cdata, one
// core at a few tens of MB/s.  Here the file streams through two pinned host buffers
// and two device buffers: the host reads chunk i+1 while chunk i is copied and parsed,
// and the device finds the row starts (non-blank lines) of a chunk with a tile count, a
// scan and a tile write, then parses one row per thread straight into the table's
// columns.  Values are rounded to FP32 exactly as fscanf's "%f" (correctly rounded,
// ties to even): a decimal m * 10^e with m < 2^53 and |e| <= 22 is converted through
// one correctly rounded double operation (m and 10^e are exact doubles), and a double
// that lands exactly between two floats is settled by the sign of the operation's
// exact remainder; any other token (more digits, larger exponents, inf, nan, hex) is
// listed for the host, which converts it with strtof and patches the table.
//
// Accepted text: fields separated by ',' with optional spaces, tabs or '\r' around
// numbers, one object per '\n'-terminated line (the last line may lack the '\n'),
// blank lines skipped (fscanf's "%f" skips them too).  A row with fewer or more than
// d fields, or a field that is not a number, is an error with the row's number.
#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/topk_b200.h"
#include "topk_internal.h"

namespace topk {

namespace {

constexpr uint32_t kTileBytes = 4096;  // row-start scan: 256 threads x 16 bytes
constexpr uint32_t kRowThreads = 256;
constexpr uint32_t kFallbackCap = 1u << 20;
constexpr uint64_t kDefaultChunk = 16ull << 20;  // bytes per pipeline buffer

enum : uint32_t { kErrNumber = 1, kErrTooFew = 2, kErrTooMany = 3, kErrShortRows = 4 };

struct Fallback {
  uint64_t row;
  uint64_t offset;  // file offset of the token
  uint32_t field;
  uint32_t pad;
};

__device__ __forceinline__ bool is_blank(char c) { return c == ' ' || c == '\t' || c == '\r'; }

// p starts a row: a character that is not white space, preceded on its line only by
// blanks (the chunk starts at a line start)
__device__ __forceinline__ bool row_start_at(const char *__restrict__ b, uint64_t p) {
  const char c = b[p];
  if (c == '\n' || is_blank(c)) return false;
  while (p > 0) {
    const char q = b[--p];
    if (q == '\n') return true;
    if (!is_blank(q)) return false;
  }
  return true;
}

__global__ void __launch_bounds__(kRowThreads)
    row_count_kernel(const char *__restrict__ buf, uint64_t len, uint32_t *__restrict__ tile_counts) {
  const uint64_t base = (uint64_t)blockIdx.x * kTileBytes + threadIdx.x * 16ull;
  uint32_t c = 0;
  for (uint32_t j = 0; j < 16; ++j)
    if (base + j < len) c += row_start_at(buf, base + j);
  c = __reduce_add_sync(0xFFFFFFFFu, c);
  __shared__ uint32_t ws[kRowThreads / 32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (uint32_t w = 0; w < kRowThreads / 32; ++w) t += ws[w];
    tile_counts[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(kRowThreads)
    row_write_kernel(const char *__restrict__ buf, uint64_t len, const uint32_t *__restrict__ tile_offsets,
                     uint32_t *__restrict__ starts, uint32_t cap) {
  const uint64_t base = (uint64_t)blockIdx.x * kTileBytes + threadIdx.x * 16ull;
  uint32_t mask = 0;
  for (uint32_t j = 0; j < 16; ++j)
    if (base + j < len && row_start_at(buf, base + j)) mask |= 1u << j;
  const uint32_t c = __popc(mask), lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = c;  // inclusive warp scan
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= (uint32_t)o) incl += v;
  }
  __shared__ uint32_t ws[kRowThreads / 32];
  if (lane == 31) ws[warp] = incl;
  __syncthreads();
  uint32_t off = tile_offsets[blockIdx.x] + incl - c;
  for (uint32_t w = 0; w < warp; ++w) off += ws[w];
  while (mask) {  // past cap some row is shorter than d fields: parse_rows_kernel reports it
    const uint32_t j = __ffs(mask) - 1;
    mask &= mask - 1;
    if (off < cap) starts[off] = (uint32_t)(base + j);
    ++off;
  }
}

// Exact powers of ten as doubles (10^0 .. 10^22 are representable).
__constant__ double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10, 1e11,
                                  1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};

// m * 10^e10 rounded once to FP32 (m < 2^53, |e10| <= 22): q = RN(m * 10^e) or RN(m /
// 10^e) in double; RN_float(q) equals RN_float(exact) unless q is a float midpoint
// (no float midpoint lies strictly between the exact value and its nearest double),
// and there the sign of the exact remainder decides.
__device__ __forceinline__ float decimal_to_float(uint64_t m, int e10) {
  const double md = (double)m;
  double q, rem;  // sign(rem) = sign(exact - q)
  if (e10 >= 0) {
    const double p = kPow10[e10];
    q = __dmul_rn(md, p);
    rem = __fma_rn(md, p, -q);
  } else {
    const double p = kPow10[-e10];
    q = __ddiv_rn(md, p);
    rem = __fma_rn(-q, p, md);
  }
  const uint64_t bits = (uint64_t)__double_as_longlong(q);
  // q in the normal float range here; the 29 bits below a float's 24-bit significand
  if ((bits & 0x1FFFFFFFull) == 0x10000000ull && rem != 0.0)
    return rem > 0.0 ? __double2float_ru(q) : __double2float_rd(q);
  return __double2float_rn(q);
}

// One numeric token at b[p..end): [+-]digits[.digits][(e|E)[+-]digits].  Returns the
// end of the token; *fast is false when the token is not of that form or is outside the
// exact range (the host converts it).
__device__ __forceinline__ uint64_t parse_number(const char *__restrict__ b, uint64_t p, uint64_t end, float *out,
                                                 bool *fast) {
  bool neg = false;
  if (p < end && (b[p] == '+' || b[p] == '-')) neg = b[p++] == '-';
  uint64_t m = 0;
  int digits = 0, e10 = 0, nd = 0;
  bool big = false;
  for (; p < end && b[p] >= '0' && b[p] <= '9'; ++p, ++nd) {
    if (m == 0 && b[p] == '0') continue;  // leading zeros
    if (digits < 19) m = m * 10 + (uint64_t)(b[p] - '0'), ++digits;
    else big = true, ++e10;
  }
  if (p < end && b[p] == '.') {
    ++p;
    for (; p < end && b[p] >= '0' && b[p] <= '9'; ++p, ++nd) {
      if (m == 0 && b[p] == '0') {
        --e10;
        continue;
      }
      if (digits < 19) m = m * 10 + (uint64_t)(b[p] - '0'), ++digits, --e10;
      else big = true;
    }
  }
  if (nd == 0) {
    *fast = false;
    return p;
  }
  if (p < end && (b[p] == 'e' || b[p] == 'E')) {
    uint64_t q = p + 1;
    bool eneg = false;
    if (q < end && (b[q] == '+' || b[q] == '-')) eneg = b[q++] == '-';
    int ev = 0, ed = 0;
    for (; q < end && b[q] >= '0' && b[q] <= '9'; ++q, ++ed)
      if (ev < 100000) ev = ev * 10 + (b[q] - '0');
    if (ed > 0) {  // otherwise the 'e' is not part of the number
      e10 += eneg ? -ev : ev;
      p = q;
    }
  }
  if (m == 0) {
    *out = neg ? -0.0f : 0.0f;
    *fast = true;
    return p;
  }
  if (big || m >= (1ull << 53) || e10 < -22 || e10 > 22) {
    *fast = false;
    return p;
  }
  const float v = decimal_to_float(m, e10);
  *out = neg ? -v : v;
  *fast = true;
  return p;
}

__global__ void parse_rows_kernel(const char *__restrict__ buf, uint64_t len, const uint32_t *__restrict__ starts,
                                  const uint32_t *__restrict__ rows_ptr, const uint64_t *__restrict__ base_ptr,
                                  uint64_t file_off, uint32_t d, float *__restrict__ table, uint64_t ld, uint64_t n,
                                  Fallback *__restrict__ fb, uint32_t *__restrict__ fb_count,
                                  unsigned long long *__restrict__ err, uint32_t cap) {
  uint32_t rows = *rows_ptr;
  const uint64_t base = *base_ptr;
  if (rows > cap) {  // rows of d fields take 2d bytes: some row of this chunk is short
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicMin(err, (unsigned long long)((base << 8) | kErrShortRows));
    rows = cap;
  }
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    const uint64_t row = base + r;
    if (row >= n) break;  // rows past n are not read (File::read_scanf_t stops at n)
    uint64_t p = starts[r];
    uint32_t code = 0;
    for (uint32_t f = 0; f < d && !code; ++f) {
      while (p < len && is_blank(buf[p])) ++p;
      const uint64_t tok = p;
      float v = 0.0f;
      bool fast = false;
      p = parse_number(buf, p, len, &v, &fast);
      if (fast && p < len && buf[p] != ',' && buf[p] != '\n' && !is_blank(buf[p])) fast = false;  // e.g. hex
      if (!fast) {  // the host converts this token; skip to its delimiter
        while (p < len && buf[p] != ',' && buf[p] != '\n') ++p;
        while (p > tok && is_blank(buf[p - 1])) --p;
        if (p == tok) {
          code = (p < len && buf[p] == '\n') || p >= len ? kErrTooFew : kErrNumber;
          break;
        }
        const uint32_t i = atomicAdd(fb_count, 1u);
        if (i < kFallbackCap) fb[i] = Fallback{row, file_off + tok, f, 0u};
      } else {
        table[(uint64_t)f * ld + row] = v;
      }
      while (p < len && is_blank(buf[p])) ++p;
      if (f + 1 < d) {
        if (p < len && buf[p] == ',') ++p;
        else code = (p >= len || buf[p] == '\n') ? kErrTooFew : kErrNumber;
      } else if (p < len && buf[p] != '\n') {
        code = buf[p] == ',' ? kErrTooMany : kErrNumber;
      }
    }
    if (code) atomicMin(err, (unsigned long long)((row << 8) | code));
  }
}

__global__ void add_rows_kernel(const uint32_t *__restrict__ rows_ptr, uint64_t *__restrict__ base_ptr) {
  *base_ptr += *rows_ptr;
}

__global__ void scatter_values_kernel(const uint64_t *__restrict__ idx, const float *__restrict__ vals, uint32_t cnt,
                                      float *__restrict__ table) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x)
    table[idx[i]] = vals[i];
}

// Row-major <-> column-major through 32 x 32 shared-memory tiles (block 32 x 8):
// reads and writes are both coalesced.  Rows on grid.x (chunks can hold millions),
// attributes on grid.y (d <= 255).
__global__ void __launch_bounds__(256)
    rows_to_cols_kernel(const float *__restrict__ src, uint32_t d, uint64_t nrows, float *__restrict__ dst,
                        uint64_t ld, uint64_t row0) {
  __shared__ float tile[32][33];
  const uint64_t r0 = (uint64_t)blockIdx.x * 32;
  const uint32_t m0 = blockIdx.y * 32;
  for (uint32_t j = threadIdx.y; j < 32; j += 8) {
    const uint64_t r = r0 + j;
    const uint32_t m = m0 + threadIdx.x;
    if (r < nrows && m < d) tile[j][threadIdx.x] = src[r * d + m];
  }
  __syncthreads();
  for (uint32_t j = threadIdx.y; j < 32; j += 8) {
    const uint32_t m = m0 + j;
    const uint64_t r = r0 + threadIdx.x;
    if (r < nrows && m < d) dst[(uint64_t)m * ld + row0 + r] = tile[threadIdx.x][j];
  }
}

__global__ void __launch_bounds__(256)
    cols_to_rows_kernel(const float *__restrict__ src, uint64_t ld, uint64_t row0, uint32_t d, uint64_t nrows,
                        float *__restrict__ dst) {
  __shared__ float tile[32][33];
  const uint64_t r0 = (uint64_t)blockIdx.x * 32;
  const uint32_t m0 = blockIdx.y * 32;
  for (uint32_t j = threadIdx.y; j < 32; j += 8) {
    const uint32_t m = m0 + j;
    const uint64_t r = r0 + threadIdx.x;
    if (r < nrows && m < d) tile[j][threadIdx.x] = src[(uint64_t)m * ld + row0 + r];
  }
  __syncthreads();
  for (uint32_t j = threadIdx.y; j < 32; j += 8) {
    const uint64_t r = r0 + j;
    const uint32_t m = m0 + threadIdx.x;
    if (r < nrows && m < d) dst[r * d + m] = tile[threadIdx.x][j];
  }
}

}  // namespace

// The loader's buffers, kept by the table handle between loads: two pinned host
// chunk buffers, two device chunk buffers with their row-start arrays, scan scratch,
// the device row counter, error word and host-conversion list, two streams (copies,
// parsing) and their events.
struct LoaderState {
  uint64_t chunk = 0, max_rows = 0;
  char *h[2] = {nullptr, nullptr};
  char *dbuf[2] = {nullptr, nullptr};
  uint32_t *tiles[2] = {nullptr, nullptr}, *offs[2] = {nullptr, nullptr}, *starts[2] = {nullptr, nullptr};
  void *temp[2] = {nullptr, nullptr};
  size_t temp_bytes = 0;
  uint64_t *base = nullptr;
  unsigned long long *err = nullptr;
  uint32_t *fb_count = nullptr;
  Fallback *fb = nullptr;
  cudaStream_t copy = nullptr, comp = nullptr;
  cudaEvent_t copied[2] = {nullptr, nullptr}, parsed[2] = {nullptr, nullptr};
  void release() {
    if (comp) cudaStreamSynchronize(comp);
    if (copy) cudaStreamSynchronize(copy);
    for (int b = 0; b < 2; ++b) {
      cudaFreeHost(h[b]);
      cudaFree(dbuf[b]);
      cudaFree(tiles[b]);
      cudaFree(offs[b]);
      cudaFree(starts[b]);
      cudaFree(temp[b]);
      if (copied[b]) cudaEventDestroy(copied[b]);
      if (parsed[b]) cudaEventDestroy(parsed[b]);
    }
    cudaFree(base);
    cudaFree(err);
    cudaFree(fb_count);
    cudaFree(fb);
    if (copy) cudaStreamDestroy(copy);
    if (comp) cudaStreamDestroy(comp);
    chunk = max_rows = 0;
    temp_bytes = 0;
    for (int b = 0; b < 2; ++b) {
      h[b] = dbuf[b] = nullptr;
      tiles[b] = offs[b] = starts[b] = nullptr;
      temp[b] = nullptr;
      copied[b] = parsed[b] = nullptr;
    }
    base = nullptr;
    err = nullptr;
    fb_count = nullptr;
    fb = nullptr;
    copy = comp = nullptr;
  }
  // buffers of chunk bytes with row arrays of max_rows; kept when they already fit
  cudaError_t reserve(uint64_t c, uint64_t rows) {
    if (chunk == c && max_rows >= rows) return cudaSuccess;
    release();
    const uint64_t max_tiles = (c + kTileBytes - 1) / kTileBytes;
    cudaError_t e = cudaSuccess;
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
      e = cudaMallocHost(&h[b], c);
      if (e == cudaSuccess) e = cudaMalloc(&dbuf[b], c);
      if (e == cudaSuccess) e = cudaMalloc(&tiles[b], (max_tiles + 1) * sizeof(uint32_t));
      if (e == cudaSuccess) e = cudaMalloc(&offs[b], (max_tiles + 1) * sizeof(uint32_t));
      if (e == cudaSuccess) e = cudaMalloc(&starts[b], rows * sizeof(uint32_t));
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&copied[b], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&parsed[b], cudaEventDisableTiming);
    }
    if (e == cudaSuccess)
      e = cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes, tiles[0], offs[0], (int)(max_tiles + 1));
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) e = cudaMalloc(&temp[b], std::max<size_t>(temp_bytes, 16));
    if (e == cudaSuccess) e = cudaMalloc(&base, sizeof(uint64_t));
    if (e == cudaSuccess) e = cudaMalloc(&err, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&fb_count, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&fb, kFallbackCap * sizeof(Fallback));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&comp, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      release();
      return e;
    }
    chunk = c;
    max_rows = rows;
    return cudaSuccess;
  }
  LoaderState() = default;
  LoaderState(const LoaderState &) = delete;
  LoaderState &operator=(const LoaderState &) = delete;
  ~LoaderState() { release(); }
};

LoaderState *loader_state_new() { return new LoaderState(); }
void loader_state_free(LoaderState *L) { delete L; }

namespace {

struct Drain {  // on every exit of a load: nothing of it stays in flight on the buffers
  LoaderState &B;
  ~Drain() {
    if (B.copy) cudaStreamSynchronize(B.copy);
    if (B.comp) cudaStreamSynchronize(B.comp);
  }
};

struct Fd {  // closes on scope exit
  int fd;
  explicit Fd(int f) : fd(f) {}
  ~Fd() {
    if (fd >= 0) close(fd);
  }
};

std::string cuda_msg(cudaError_t e, const char *what) { return std::string(what) + ": " + cudaGetErrorString(e); }

// read exactly want bytes unless the file ends; returns the count or -1
int64_t read_full(int fd, char *dst, uint64_t want) {
  uint64_t got = 0;
  while (got < want) {
    const ssize_t r = read(fd, dst + got, (size_t)std::min<uint64_t>(want - got, 1ull << 30));
    if (r < 0) {
      if (errno == EINTR) continue;
      return -1;
    }
    if (r == 0) break;
    got += (uint64_t)r;
  }
  return (int64_t)got;
}

bool pread_full(int fd, char *dst, uint64_t want, uint64_t off, uint64_t *got) {
  *got = 0;
  while (*got < want) {
    const ssize_t r = pread(fd, dst + *got, (size_t)(want - *got), (off_t)(off + *got));
    if (r < 0) {
      if (errno == EINTR) continue;
      return false;
    }
    if (r == 0) break;
    *got += (uint64_t)r;
  }
  return true;
}

// pread of [off, off + bytes) split over up to 8 threads (page-cache copies scale
// with threads; one thread reads at a few GB/s)
bool parallel_pread(int fd, char *dst, uint64_t bytes, uint64_t off) {
  const uint64_t piece = 4ull << 20;
  const unsigned nt = (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>({8, (bytes + piece - 1) / piece, std::max(1u, std::thread::hardware_concurrency())}));
  if (nt == 1) {
    uint64_t got = 0;
    return pread_full(fd, dst, bytes, off, &got) && got == bytes;
  }
  const uint64_t per = (bytes + nt - 1) / nt;
  std::vector<std::thread> th;
  std::vector<int> ok(nt, 0);
  for (unsigned t = 0; t < nt; ++t)
    th.emplace_back([&, t]() {
      const uint64_t a = std::min<uint64_t>(bytes, (uint64_t)t * per), b = std::min<uint64_t>(bytes, a + per);
      uint64_t got = 0;
      ok[t] = pread_full(fd, dst + a, b - a, off + a, &got) && got == b - a;
    });
  for (auto &x : th) x.join();
  for (int v : ok)
    if (!v) return false;
  return true;
}

}  // namespace

int csv_shape(const char *path, uint64_t *n, uint64_t *d, std::string *msg) {
  // File<T>::count (input/File.h:108-132): d = 1 + the commas of the first line,
  // n = the newlines of the file
  const int fd = open(path, O_RDONLY);
  if (fd < 0) {
    *msg = std::string("cannot open ") + path + ": " + strerror(errno);
    return TOPK_ERR_ARG;
  }
  std::vector<char> buf(16u << 20);
  uint64_t nn = 0, dd = 1;
  bool first = true;
  for (;;) {
    const int64_t r = read_full(fd, buf.data(), buf.size());
    if (r < 0) {
      close(fd);
      *msg = std::string("read failed: ") + strerror(errno);
      return TOPK_ERR_ARG;
    }
    if (r == 0) break;
    for (int64_t i = 0; i < r; ++i) {
      const char c = buf[(size_t)i];
      if (first && c == ',') ++dd;
      if (c == '\n') ++nn, first = false;
    }
  }
  close(fd);
  *n = nn;
  *d = dd;
  return TOPK_OK;
}

int load_csv_device(LoaderState *L, const char *path, float *table, uint64_t ld, uint32_t d, uint64_t n,
                    int num_sms, uint64_t chunk_bytes, uint64_t stats[4], std::string *msg) {
  if (chunk_bytes == 0) chunk_bytes = kDefaultChunk;
  chunk_bytes = std::max<uint64_t>(chunk_bytes, 1024);
  if (chunk_bytes > (1ull << 31)) chunk_bytes = 1ull << 31;
  chunk_bytes = (chunk_bytes + 15) & ~15ull;
  Fd F(open(path, O_RDONLY));
  if (F.fd < 0) {
    *msg = std::string("cannot open ") + path + ": " + strerror(errno);
    return TOPK_ERR_ARG;
  }
  struct stat st;
  if (fstat(F.fd, &st) != 0) {
    *msg = std::string("cannot stat ") + path;
    return TOPK_ERR_ARG;
  }
  const uint64_t fsize = (uint64_t)st.st_size;
  // a row of d fields takes at least 2d bytes ("x," ... "x\n")
  const uint64_t max_rows = chunk_bytes / (2ull * d) + 2;
  LoaderState &B = *L;
  Drain drain{B};
  cudaError_t e = B.reserve(chunk_bytes, max_rows);
  if (e == cudaSuccess) e = cudaMemsetAsync(B.base, 0, sizeof(uint64_t), B.comp);
  if (e == cudaSuccess) e = cudaMemsetAsync(B.err, 0xFF, sizeof(unsigned long long), B.comp);
  if (e == cudaSuccess) e = cudaMemsetAsync(B.fb_count, 0, sizeof(uint32_t), B.comp);
  if (e == cudaSuccess) e = cudaStreamSynchronize(B.comp);
  if (e != cudaSuccess) {
    *msg = cuda_msg(e, "loader setup");
    return e == cudaErrorMemoryAllocation ? TOPK_ERR_OOM : TOPK_ERR_CUDA;
  }
  const uint32_t cap = (uint32_t)std::min<uint64_t>(B.max_rows, 0xFFFFFFFFull);
  const int grid = num_sms * 8;
  bool used[2] = {false, false};
  int chunks = 0;
  // copy h[b][0, len) to the device and parse it (rows start at the device's row count)
  auto enqueue = [&](int b, uint64_t len, uint64_t off) -> cudaError_t {
    cudaError_t r = cudaSuccess;
    if (used[b]) r = cudaStreamWaitEvent(B.copy, B.parsed[b], 0);  // device buffer b parsed two chunks ago
    if (r == cudaSuccess) r = cudaMemcpyAsync(B.dbuf[b], B.h[b], len, cudaMemcpyHostToDevice, B.copy);
    if (r == cudaSuccess) r = cudaEventRecord(B.copied[b], B.copy);
    if (r == cudaSuccess) r = cudaStreamWaitEvent(B.comp, B.copied[b], 0);
    const uint32_t tiles = (uint32_t)((len + kTileBytes - 1) / kTileBytes);
    if (r == cudaSuccess) {
      row_count_kernel<<<tiles, kRowThreads, 0, B.comp>>>(B.dbuf[b], len, B.tiles[b]);
      r = cudaMemsetAsync(B.tiles[b] + tiles, 0, sizeof(uint32_t), B.comp);
    }
    size_t tb = B.temp_bytes;
    if (r == cudaSuccess) r = cub::DeviceScan::ExclusiveSum(B.temp[b], tb, B.tiles[b], B.offs[b], (int)tiles + 1, B.comp);
    if (r == cudaSuccess) {
      row_write_kernel<<<tiles, kRowThreads, 0, B.comp>>>(B.dbuf[b], len, B.offs[b], B.starts[b], cap);
      parse_rows_kernel<<<grid, 128, 0, B.comp>>>(B.dbuf[b], len, B.starts[b], B.offs[b] + tiles, B.base, off, d,
                                                 table, ld, n, B.fb, B.fb_count, B.err, cap);
      add_rows_kernel<<<1, 1, 0, B.comp>>>(B.offs[b] + tiles, B.base);
      r = cudaEventRecord(B.parsed[b], B.comp);
    }
    used[b] = true;
    ++chunks;
    return r;
  };
  uint64_t file_off = 0, carry = 0, read_pos = 0;  // carry: an unfinished line, at carry_src
  const char *carry_src = nullptr;
  for (int b = 0;; b ^= 1) {
    if (used[b]) {  // host buffer b was copied two chunks ago
      e = cudaEventSynchronize(B.copied[b]);
      if (e != cudaSuccess) break;
    }
    if (carry) memcpy(B.h[b], carry_src, carry);
    const uint64_t got = std::min<uint64_t>(chunk_bytes - carry, fsize - read_pos);
    if (got && !parallel_pread(F.fd, B.h[b] + carry, got, read_pos)) {
      *msg = std::string("read failed: ") + strerror(errno);
      return TOPK_ERR_ARG;
    }
    read_pos += got;
    const bool eof = read_pos == fsize;
    const uint64_t len = carry + (uint64_t)got;
    uint64_t cut = len;  // whole lines; at the end of the file, everything (the last '\n' may be missing)
    if (!eof) {
      while (cut > 0 && B.h[b][cut - 1] != '\n') --cut;
      if (cut == 0) {
        *msg = "a line is longer than the load chunk (" + std::to_string(chunk_bytes) + " bytes)";
        return TOPK_ERR_UNSUPPORTED;
      }
    }
    if (cut > 0) {
      e = enqueue(b, cut, file_off);
      if (e != cudaSuccess) break;
    }
    file_off += cut;
    carry = len - cut;
    carry_src = B.h[b] + cut;  // not overwritten before the next chunk copies it out
    if (eof) break;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(B.comp);
  uint64_t rows = 0;
  unsigned long long err = 0;
  uint32_t nfb = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&rows, B.base, sizeof(rows), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&err, B.err, sizeof(err), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&nfb, B.fb_count, sizeof(nfb), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    *msg = cuda_msg(e, "loader");
    return TOPK_ERR_CUDA;
  }
  if (err != ~0ull) {
    const uint64_t row = err >> 8;
    const uint32_t code = (uint32_t)(err & 0xFF);
    *msg = code == kErrShortRows
               ? "rows with fewer than " + std::to_string(d) + " fields after row " + std::to_string(row)
               : "row " + std::to_string(row + 1) + ": " +
                     (code == kErrTooFew   ? "fewer than " + std::to_string(d) + " fields"
                      : code == kErrTooMany ? "more than " + std::to_string(d) + " fields"
                                            : "not a number");
    return TOPK_ERR_ARG;
  }
  if (rows < n) {
    *msg = "the file holds " + std::to_string(rows) + " rows, the table " + std::to_string(n);
    return TOPK_ERR_ARG;
  }
  if (nfb > kFallbackCap) {
    *msg = std::to_string(nfb) + " values outside the device parser's exact range (at most " +
           std::to_string(kFallbackCap) + ")";
    return TOPK_ERR_UNSUPPORTED;
  }
  if (nfb > 0) {  // host conversion of the listed tokens (strtof, as fscanf's %f)
    std::vector<Fallback> fb(nfb);
    e = cudaMemcpy(fb.data(), B.fb, nfb * sizeof(Fallback), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      *msg = cuda_msg(e, "loader fallbacks");
      return TOPK_ERR_CUDA;
    }
    std::vector<uint64_t> idx(nfb);
    std::vector<float> val(nfb);
    std::vector<char> tok(4096);
    for (uint32_t i = 0; i < nfb; ++i) {
      uint64_t got = 0;
      if (!pread_full(F.fd, tok.data(), tok.size() - 1, fb[i].offset, &got)) {
        *msg = "re-read failed";
        return TOPK_ERR_ARG;
      }
      tok[got] = 0;
      size_t L = 0;
      while (L < got && tok[L] != ',' && tok[L] != '\n') ++L;
      if (L == got && got == tok.size() - 1) {
        *msg = "row " + std::to_string(fb[i].row + 1) + ": a field longer than 4095 bytes";
        return TOPK_ERR_UNSUPPORTED;
      }
      while (L > 0 && (tok[L - 1] == ' ' || tok[L - 1] == '\t' || tok[L - 1] == '\r')) --L;
      tok[L] = 0;
      char *endp = nullptr;
      errno = 0;
      const float v = strtof(tok.data(), &endp);
      if (endp != tok.data() + L || L == 0) {
        *msg = "row " + std::to_string(fb[i].row + 1) + ": not a number: " + std::string(tok.data(), L);
        return TOPK_ERR_ARG;
      }
      idx[i] = (uint64_t)fb[i].field * ld + fb[i].row;
      val[i] = v;
    }
    uint64_t *didx = nullptr;
    float *dval = nullptr;
    e = cudaMalloc(&didx, nfb * sizeof(uint64_t));
    if (e == cudaSuccess) e = cudaMalloc(&dval, nfb * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(didx, idx.data(), nfb * sizeof(uint64_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dval, val.data(), nfb * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
      scatter_values_kernel<<<std::min<uint32_t>((nfb + 255) / 256, 1024), 256, 0, B.comp>>>(didx, dval, nfb, table);
      e = cudaStreamSynchronize(B.comp);
    }
    cudaFree(didx);
    cudaFree(dval);
    if (e != cudaSuccess) {
      *msg = cuda_msg(e, "loader fallbacks");
      return TOPK_ERR_CUDA;
    }
  }
  if (stats) {
    stats[0] = file_off;
    stats[1] = rows;
    stats[2] = nfb;
    stats[3] = (uint64_t)chunks;
  }
  return TOPK_OK;
}

// ------------------------------------------------------------------ writers
// The reference's File<T>::store (input/File.h:405-431) writes each object as one line
// of "%f" fields separated by ',' (write_printf_t); save_csv writes the same text for
// every d (the reference's writer handles even d only, File.h:357-403).
int save_csv(const char *path, const float *table, uint64_t ld, uint32_t d, uint64_t n, std::string *msg) {
  FILE *f = fopen(path, "wb");
  if (!f) {
    *msg = std::string("cannot create ") + path + ": " + strerror(errno);
    return TOPK_ERR_ARG;
  }
  const uint64_t block = 1u << 16;  // rows per formatting block
  const unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  std::vector<float> cols((size_t)d * block * nt);
  std::vector<std::string> text(nt);
  int rc = TOPK_OK;
  for (uint64_t r0 = 0; r0 < n && rc == TOPK_OK; r0 += block * nt) {
    const uint64_t rows = std::min<uint64_t>(block * nt, n - r0);
    cudaError_t e = cudaMemcpy2D(cols.data(), rows * sizeof(float), table + r0, ld * sizeof(float),
                                 rows * sizeof(float), d, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      *msg = cuda_msg(e, "save_csv");
      rc = TOPK_ERR_CUDA;
      break;
    }
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t) {
      th.emplace_back([&, t]() {
        std::string &out = text[t];
        out.clear();
        char tmp[64];
        const uint64_t a = std::min<uint64_t>(rows, t * block), b = std::min<uint64_t>(rows, (t + 1) * block);
        for (uint64_t i = a; i < b; ++i) {
          for (uint32_t m = 0; m < d; ++m) {
            const int k = snprintf(tmp, sizeof(tmp), m + 1 < d ? "%f," : "%f\n", (double)cols[(size_t)m * rows + i]);
            out.append(tmp, (size_t)k);
          }
        }
      });
    }
    for (auto &x : th) x.join();
    for (unsigned t = 0; t < nt; ++t)
      if (!text[t].empty() && fwrite(text[t].data(), 1, text[t].size(), f) != text[t].size()) {
        *msg = "write failed";
        rc = TOPK_ERR_ARG;
        break;
      }
  }
  if (fclose(f) != 0 && rc == TOPK_OK) {
    *msg = "close failed";
    rc = TOPK_ERR_ARG;
  }
  return rc;
}

// Binary column-major table file: a 64-byte header, then the d columns of n FP32
// values each (column m at byte 64 + 4*n*m).
namespace {
struct BinHeader {
  char magic[8];     // "TOPKCOL1"
  uint32_t version;  // 1
  uint32_t elem;     // 4 (FP32)
  uint64_t n, d;
  uint64_t reserved[4];
};
static_assert(sizeof(BinHeader) == 64, "header is 64 bytes");
const char kMagic[8] = {'T', 'O', 'P', 'K', 'C', 'O', 'L', '1'};
}  // namespace

int binary_shape(const char *path, uint64_t *n, uint64_t *d, std::string *msg) {
  const int fd = open(path, O_RDONLY);
  if (fd < 0) {
    *msg = std::string("cannot open ") + path + ": " + strerror(errno);
    return TOPK_ERR_ARG;
  }
  BinHeader hd;
  uint64_t got = 0;
  const bool ok = pread_full(fd, reinterpret_cast<char *>(&hd), sizeof(hd), 0, &got) && got == sizeof(hd);
  struct stat st;
  const bool sized = fstat(fd, &st) == 0;
  close(fd);
  if (!ok || memcmp(hd.magic, kMagic, 8) != 0 || hd.version != 1 || hd.elem != 4) {
    *msg = std::string(path) + " is not a TOPKCOL1 table file";
    return TOPK_ERR_ARG;
  }
  if (!sized || (uint64_t)st.st_size < sizeof(hd) + 4 * hd.n * hd.d) {
    *msg = std::string(path) + " is shorter than its header says";
    return TOPK_ERR_ARG;
  }
  *n = hd.n;
  *d = hd.d;
  return TOPK_OK;
}

int save_binary(const char *path, const float *table, uint64_t ld, uint32_t d, uint64_t n, std::string *msg) {
  FILE *f = fopen(path, "wb");
  if (!f) {
    *msg = std::string("cannot create ") + path + ": " + strerror(errno);
    return TOPK_ERR_ARG;
  }
  BinHeader hd{};
  memcpy(hd.magic, kMagic, 8);
  hd.version = 1;
  hd.elem = 4;
  hd.n = n;
  hd.d = d;
  int rc = fwrite(&hd, sizeof(hd), 1, f) == 1 ? TOPK_OK : TOPK_ERR_ARG;
  const uint64_t chunk = 16u << 20;  // floats per copy
  float *h = nullptr;
  if (rc == TOPK_OK && cudaMallocHost(&h, chunk * sizeof(float)) != cudaSuccess) rc = TOPK_ERR_OOM;
  for (uint32_t m = 0; m < d && rc == TOPK_OK; ++m)
    for (uint64_t r0 = 0; r0 < n && rc == TOPK_OK; r0 += chunk) {
      const uint64_t c = std::min(chunk, n - r0);
      if (cudaMemcpy(h, table + (uint64_t)m * ld + r0, c * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = TOPK_ERR_CUDA;
      else if (fwrite(h, sizeof(float), c, f) != c)
        rc = TOPK_ERR_ARG;
    }
  cudaFreeHost(h);
  if (fclose(f) != 0 && rc == TOPK_OK) rc = TOPK_ERR_ARG;
  if (rc != TOPK_OK) *msg = std::string("writing ") + path + " failed";
  return rc;
}

// Reads the columns through two pinned buffers: the read of one chunk overlaps the
// copy of the other.
int load_binary_device(LoaderState *L, const char *path, float *table, uint64_t ld, uint32_t d, uint64_t n,
                       std::string *msg) {
  uint64_t fn = 0, fd_ = 0;
  int rc = binary_shape(path, &fn, &fd_, msg);
  if (rc != TOPK_OK) return rc;
  if (fn != n || fd_ != d) {
    *msg = "the file holds " + std::to_string(fn) + " x " + std::to_string(fd_) + ", the table " +
           std::to_string(n) + " x " + std::to_string(d);
    return TOPK_ERR_ARG;
  }
  Fd F(open(path, O_RDONLY));
  if (F.fd < 0) {
    *msg = std::string("cannot open ") + path;
    return TOPK_ERR_ARG;
  }
  LoaderState &B = *L;
  Drain drain{B};
  cudaError_t e = B.chunk ? cudaSuccess : B.reserve(kDefaultChunk, 2);
  if (e != cudaSuccess) {
    *msg = cuda_msg(e, "loader setup");
    return e == cudaErrorMemoryAllocation ? TOPK_ERR_OOM : TOPK_ERR_CUDA;
  }
  const uint64_t chunk = B.chunk / sizeof(float);  // floats per buffer
  bool used[2] = {false, false};
  int b = 0;
  for (uint32_t m = 0; m < d && e == cudaSuccess; ++m)
    for (uint64_t r0 = 0; r0 < n && e == cudaSuccess; r0 += chunk, b ^= 1) {
      const uint64_t c = std::min(chunk, n - r0);
      if (used[b]) e = cudaEventSynchronize(B.copied[b]);  // the copy out of buffer b is done
      if (e != cudaSuccess) break;
      if (!parallel_pread(F.fd, B.h[b], c * sizeof(float), sizeof(BinHeader) + 4 * ((uint64_t)m * n + r0))) {
        cudaStreamSynchronize(B.copy);
        *msg = std::string("reading ") + path + " failed";
        return TOPK_ERR_ARG;
      }
      e = cudaMemcpyAsync(table + (uint64_t)m * ld + r0, B.h[b], c * sizeof(float), cudaMemcpyHostToDevice, B.copy);
      if (e == cudaSuccess) e = cudaEventRecord(B.copied[b], B.copy);
      used[b] = true;
    }
  if (e == cudaSuccess) e = cudaStreamSynchronize(B.copy);
  if (e != cudaSuccess) {
    *msg = cuda_msg(e, "load_binary");
    return TOPK_ERR_CUDA;
  }
  return TOPK_OK;
}

// ------------------------------------------------------------ row-major tables
// The reference's TPAr keeps the table row-major (cpu/TPAr.h, cdata[i*d + m]) and
// normalises it in place (common/common.h:63-92, the same arithmetic per attribute as
// normalize_transpose).  Row-major host tables go through the pipeline buffers: a
// strided 2D copy of a block of rows into a device buffer, then a tiled transpose
// into the column-major table; the next block's copy overlaps this block's transpose.
namespace {
int rowmajor_prepare(LoaderState &B, std::string *msg) {
  cudaError_t e = B.chunk >= kDefaultChunk ? cudaSuccess : B.reserve(kDefaultChunk, std::max<uint64_t>(B.max_rows, 2));
  if (e != cudaSuccess) {
    *msg = cuda_msg(e, "row-major staging");
    return e == cudaErrorMemoryAllocation ? TOPK_ERR_OOM : TOPK_ERR_CUDA;
  }
  return TOPK_OK;
}
}  // namespace

namespace {
// rows x width floats between strided host arrays, split over up to 8 threads
void copy_rows(float *dst, uint64_t dst_stride, const float *src, uint64_t src_stride, uint64_t rows,
               uint64_t width) {
  const unsigned nt = (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>({8, rows * width / (1u << 18) + 1, std::max(1u, std::thread::hardware_concurrency())}));
  auto part = [&](uint64_t a, uint64_t b) {
    if (dst_stride == width && src_stride == width) {
      memcpy(dst + a * width, src + a * width, (b - a) * width * sizeof(float));
      return;
    }
    for (uint64_t r = a; r < b; ++r) memcpy(dst + r * dst_stride, src + r * src_stride, width * sizeof(float));
  };
  if (nt == 1) {
    part(0, rows);
    return;
  }
  std::vector<std::thread> th;
  const uint64_t per = (rows + nt - 1) / nt;
  for (unsigned t = 0; t < nt; ++t) {
    const uint64_t a = std::min<uint64_t>(rows, t * per), b = std::min<uint64_t>(rows, a + per);
    th.emplace_back(part, a, b);
  }
  for (auto &x : th) x.join();
}
}  // namespace

// Upload: block i's rows are packed into pinned buffer i % 2 by host threads while
// block i-1 is copied and transposed; download runs the same pipeline backwards.
int upload_rowmajor_device(LoaderState *L, const float *host, uint64_t row_stride, float *table, uint64_t ld,
                           uint32_t d, uint64_t n, std::string *msg) {
  LoaderState &B = *L;
  Drain drain{B};
  int rc = rowmajor_prepare(B, msg);
  if (rc != TOPK_OK) return rc;
  const uint64_t per = B.chunk / (4ull * d);  // rows per buffer
  bool used[2] = {false, false};
  cudaError_t e = cudaSuccess;
  int b = 0;
  for (uint64_t r0 = 0; r0 < n && e == cudaSuccess; r0 += per, b ^= 1) {
    const uint64_t rows = std::min(per, n - r0);
    float *hb = reinterpret_cast<float *>(B.h[b]), *stage = reinterpret_cast<float *>(B.dbuf[b]);
    if (used[b]) e = cudaEventSynchronize(B.copied[b]);  // pinned buffer b copied out
    if (e != cudaSuccess) break;
    copy_rows(hb, d, host + r0 * row_stride, row_stride, rows, d);
    if (used[b]) e = cudaStreamWaitEvent(B.copy, B.parsed[b], 0);  // device buffer b transposed
    if (e == cudaSuccess) e = cudaMemcpyAsync(stage, hb, rows * d * sizeof(float), cudaMemcpyHostToDevice, B.copy);
    if (e == cudaSuccess) e = cudaEventRecord(B.copied[b], B.copy);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(B.comp, B.copied[b], 0);
    if (e == cudaSuccess) {
      rows_to_cols_kernel<<<dim3((unsigned)((rows + 31) / 32), (d + 31) / 32), dim3(32, 8), 0, B.comp>>>(
          stage, d, rows, table, ld, r0);
      e = cudaEventRecord(B.parsed[b], B.comp);
    }
    used[b] = true;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(B.comp);
  if (e != cudaSuccess) {
    *msg = cuda_msg(e, "upload_rowmajor");
    return TOPK_ERR_CUDA;
  }
  return TOPK_OK;
}

int download_rowmajor_device(LoaderState *L, float *host, uint64_t row_stride, const float *table, uint64_t ld,
                             uint32_t d, uint64_t n, std::string *msg) {
  LoaderState &B = *L;
  Drain drain{B};
  int rc = rowmajor_prepare(B, msg);
  if (rc != TOPK_OK) return rc;
  const uint64_t per = B.chunk / (4ull * d);
  cudaError_t e = cudaSuccess;
  int64_t pending = -1;  // block waiting in its pinned buffer to be unpacked
  int pb = 0;
  auto unpack = [&]() -> cudaError_t {
    if (pending < 0) return cudaSuccess;
    cudaError_t r = cudaEventSynchronize(B.copied[pb]);
    if (r != cudaSuccess) return r;
    const uint64_t r0 = (uint64_t)pending * per, rows = std::min(per, n - r0);
    copy_rows(host + r0 * row_stride, row_stride, reinterpret_cast<const float *>(B.h[pb]), d, rows, d);
    pending = -1;
    return cudaSuccess;
  };
  int b = 0;
  for (uint64_t r0 = 0, blk = 0; r0 < n && e == cudaSuccess; r0 += per, ++blk, b ^= 1) {
    const uint64_t rows = std::min(per, n - r0);
    float *stage = reinterpret_cast<float *>(B.dbuf[b]);
    // buffers b were last used by block blk - 2, unpacked before block blk - 1 was queued
    cols_to_rows_kernel<<<dim3((unsigned)((rows + 31) / 32), (d + 31) / 32), dim3(32, 8), 0, B.comp>>>(
        table, ld, r0, d, rows, stage);
    e = cudaEventRecord(B.parsed[b], B.comp);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(B.copy, B.parsed[b], 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(B.h[b], stage, rows * d * sizeof(float), cudaMemcpyDeviceToHost, B.copy);
    if (e == cudaSuccess) e = cudaEventRecord(B.copied[b], B.copy);
    if (e == cudaSuccess) e = unpack();  // the previous block, while this one is in flight
    pending = (int64_t)blk;
    pb = b;
  }
  if (e == cudaSuccess) e = unpack();
  if (e != cudaSuccess) {
    *msg = cuda_msg(e, "download_rowmajor");
    return TOPK_ERR_CUDA;
  }
  return TOPK_OK;
}

}  // namespace topk
