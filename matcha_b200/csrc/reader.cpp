// Subtomogram / CTF-weight file decode for the batch reader (host code, no GPU).
//
// Reference behaviour restated here (paths inside swing-research/Matcha):
//   load_subtomogram_cpu      src/matcha/utils/io_utils.py:229-238  mrcfile data as float32,
//                                                                    C order (z, y, x)
//   load_ctf_relion5_cpu      src/matcha/utils/io_utils.py:240-253  the same, cropped to
//                                                                    [:nz/2, :, :nz/2+1]
//   _read_worker / cpu_reader src/matcha/utils/run_utils.py:23-41, 430-611  a thread pool
//                                                                    reads each file; a file
//                                                                    that fails is skipped
//
// The MRC2014 layout: a 1024-byte header of 32-bit words (NX, NY, NZ, MODE at bytes 0-15,
// NSYMBT, the extended header's length, at byte 92, the machine stamp at byte 212: 0x44 or
// 0x41 first for little-endian, 0x11 for big-endian), the extended header, then the voxels
// with x fastest.  Modes decoded: 0 int8, 1 int16, 2 float32, 6 uint16, 12 float16.
//
// Worker threads claim files from an atomic counter and pread each straight into its slot of
// the caller's (pinned) batch buffer: a float32 file in native byte order whose crop is whole
// planes is read with no intermediate copy; other modes and byte orders go through a
// per-thread buffer and are converted.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <atomic>
#include <cerrno>
#include <cstdint>
#include <cstring>
#include <new>
#include <system_error>
#include <thread>
#include <vector>

#include "matcha_b200.h"

struct mtb_reader {
  int n_threads;
};

namespace {

struct Header {
  int64_t nx, ny, nz;
  int mode;
  int esize;
  bool swap;
  int64_t offset;
};

uint32_t load32(const unsigned char* p, bool swap) {
  uint32_t v;
  std::memcpy(&v, p, 4);
  return swap ? __builtin_bswap32(v) : v;
}

int mode_size(int mode) {
  switch (mode) {
    case 0: return 1;
    case 1: return 2;
    case 2: return 4;
    case 6: return 2;
    case 12: return 2;
    default: return 0;
  }
}

// IEEE 754 binary16 -> binary32 from the bit fields (sign, 5-bit exponent, 10-bit fraction).
float half_to_float(uint16_t h) {
  const uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
  uint32_t exp = (h >> 10) & 0x1fu, frac = h & 0x3ffu, bits;
  if (exp == 0) {
    if (frac == 0) {
      bits = sign;
    } else {  // subnormal: shift the fraction up to a normal number
      int e = 113;  // 127 - 15 + 1
      while (!(frac & 0x400u)) {
        frac <<= 1;
        --e;
      }
      bits = sign | ((uint32_t)e << 23) | ((frac & 0x3ffu) << 13);
    }
  } else if (exp == 31) {
    bits = sign | 0x7f800000u | (frac << 13);
  } else {
    bits = sign | ((exp + 112) << 23) | (frac << 13);
  }
  float f;
  std::memcpy(&f, &bits, 4);
  return f;
}

bool pread_all(int fd, void* buf, size_t n, int64_t off) {
  char* p = static_cast<char*>(buf);
  while (n > 0) {
    const ssize_t r = pread(fd, p, n, (off_t)off);
    if (r < 0) {
      if (errno == EINTR) continue;
      return false;
    }
    if (r == 0) return false;
    p += r;
    n -= (size_t)r;
    off += r;
  }
  return true;
}

int parse_header(int fd, int64_t fsize, Header* h) {
  unsigned char hdr[1024];
  if (fsize < 1024 || !pread_all(fd, hdr, sizeof(hdr), 0)) return MTB_READ_HEADER;
  bool swap;
  if (hdr[212] == 0x44 || hdr[212] == 0x41) {
    swap = false;
  } else if (hdr[212] == 0x11) {
    swap = true;
  } else {  // no valid machine stamp: take the byte order in which the mode is one we know
    swap = mode_size((int)load32(hdr + 12, false)) == 0 && mode_size((int)load32(hdr + 12, true)) != 0;
  }
  h->swap = swap;
  h->nx = (int32_t)load32(hdr, swap);
  h->ny = (int32_t)load32(hdr + 4, swap);
  h->nz = (int32_t)load32(hdr + 8, swap);
  h->mode = (int32_t)load32(hdr + 12, swap);
  const int64_t nsymbt = (int32_t)load32(hdr + 92, swap);
  h->esize = mode_size(h->mode);
  if (h->esize == 0 || h->nx <= 0 || h->ny <= 0 || h->nz <= 0 || nsymbt < 0) return MTB_READ_HEADER;
  h->offset = 1024 + nsymbt;
  if (fsize < h->offset + h->nx * h->ny * h->nz * h->esize) return MTB_READ_SHORT;
  return MTB_READ_OK;
}

void convert(const unsigned char* src, int64_t n, const Header& h, float* dst) {
  switch (h.mode) {
    case 0:
      for (int64_t i = 0; i < n; ++i) dst[i] = (float)(int8_t)src[i];
      break;
    case 1:
    case 6:
    case 12:
      for (int64_t i = 0; i < n; ++i) {
        uint16_t v;
        std::memcpy(&v, src + 2 * i, 2);
        if (h.swap) v = __builtin_bswap16(v);
        dst[i] = h.mode == 1 ? (float)(int16_t)v : h.mode == 6 ? (float)v : half_to_float(v);
      }
      break;
    default:
      for (int64_t i = 0; i < n; ++i) {
        uint32_t v;
        std::memcpy(&v, src + 4 * i, 4);
        if (h.swap) v = __builtin_bswap32(v);
        std::memcpy(dst + i, &v, 4);
      }
  }
}

// Decode [0, cz) x [0, cy) x [0, cx) of the file into dst (cz * cy * cx floats).
int decode(const char* path, int64_t nz, int64_t ny, int64_t nx, int64_t cz, int64_t cy, int64_t cx, float* dst,
           std::vector<unsigned char>& scratch) {
  const int fd = open(path, O_RDONLY | O_CLOEXEC);
  if (fd < 0) return MTB_READ_OPEN;
  struct stat sb;
  int rc = fstat(fd, &sb) == 0 ? MTB_READ_OK : MTB_READ_OPEN;
  Header h{};
  if (rc == MTB_READ_OK) rc = parse_header(fd, (int64_t)sb.st_size, &h);
  if (rc == MTB_READ_OK && (h.nz != nz || h.ny != ny || h.nx != nx)) rc = MTB_READ_SHAPE;
  if (rc == MTB_READ_OK) {
    const int64_t plane = ny * nx;
    if (h.mode == 2 && !h.swap && cy == ny && cx == nx) {
      if (!pread_all(fd, dst, (size_t)(cz * plane * 4), h.offset)) rc = MTB_READ_SHORT;
    } else {
      // plane by plane: read the rows [0, cy) of plane z, keep columns [0, cx)
      const size_t bytes = (size_t)(cy * nx * h.esize);
      if (scratch.size() < bytes) scratch.resize(bytes);
      std::vector<float> row((size_t)nx);
      for (int64_t z = 0; z < cz && rc == MTB_READ_OK; ++z) {
        if (!pread_all(fd, scratch.data(), bytes, h.offset + z * plane * h.esize)) {
          rc = MTB_READ_SHORT;
          break;
        }
        for (int64_t y = 0; y < cy; ++y) {
          float* out = dst + (z * cy + y) * cx;
          if (cx == nx) {
            convert(scratch.data() + y * nx * h.esize, nx, h, out);
          } else {
            convert(scratch.data() + y * nx * h.esize, cx, h, row.data());
            std::memcpy(out, row.data(), (size_t)cx * sizeof(float));
          }
        }
      }
    }
  }
  close(fd);
  return rc;
}

}  // namespace

extern "C" int mtb_reader_create(int n_threads, mtb_reader** out) {
  if (!out || n_threads < 0) return MTB_ERR_ARG;
  if (n_threads == 0) {
    const unsigned hc = std::thread::hardware_concurrency();
    n_threads = hc ? (int)hc : 1;
  }
  *out = new (std::nothrow) mtb_reader{n_threads};
  return *out ? MTB_OK : MTB_ERR_OOM;
}

extern "C" int mtb_reader_destroy(mtb_reader* r) {
  delete r;
  return MTB_OK;
}

extern "C" int mtb_read_mrc(mtb_reader* r, const char* const* paths, int n, int nz, int ny, int nx, int cz, int cy,
                            int cx, float* dst, int* status) {
  if (!r || n < 0) return MTB_ERR_ARG;
  if (n == 0) return MTB_OK;
  if (!paths || !dst || !status) return MTB_ERR_ARG;
  if (nz <= 0 || ny <= 0 || nx <= 0 || cz <= 0 || cy <= 0 || cx <= 0 || cz > nz || cy > ny || cx > nx)
    return MTB_ERR_ARG;
  const int64_t per = (int64_t)cz * cy * cx;
  std::atomic<int> next{0};
  auto work = [&]() {
    std::vector<unsigned char> scratch;
    for (int i = next++; i < n; i = next++) {
      status[i] = paths[i] ? decode(paths[i], nz, ny, nx, cz, cy, cx, dst + per * i, scratch) : MTB_READ_OPEN;
    }
  };
  const int nt = r->n_threads < n ? r->n_threads : n;
  std::vector<std::thread> pool;
  try {
    pool.reserve((size_t)(nt > 0 ? nt - 1 : 0));
    for (int t = 1; t < nt; ++t) pool.emplace_back(work);
  } catch (const std::exception&) {
    // fewer threads than asked for: the ones started, and this one, share the files
  }
  work();
  for (auto& t : pool) t.join();
  return MTB_OK;
}
