// Binary checkpoint files of the order parameter (host code only).
//
// The reference keeps no resumable state: its only copies are the in-memory
// temp_stor_data / reset_data pair (src/fft_fftw_slab.cpp:1891-1925) and the
// text dumps (src/dump_text.cpp:361-400, six significant digits).  A
// checkpoint here is the device state of one instance as it is stepped:
//
//   header (256 bytes, little-endian)
//     0   char[8]   "PFDDCKP1"
//     8   u32       format version (2)
//     12  u32       header size (256)
//     16  i32[8]    nx, ny, nz, n_slip, fields carried, precision, imag mode, advanced
//     48  u64       field bytes, 56 u64 carrier bytes
//     64  f64[18]   sigma[3][3], dsigma[3][3] (units of mu) of the device
//     208 u64       steps recorded by the writer (informational)
//     216 u64       FNV-1a 64 of the payload
//     224 u64       FNV-1a 64 of header bytes 0..223
//     232 ...       zero
//   payload: the fields (fields carried x N values of the compute precision,
//   reference site order), then the Nyquist carrier of Im xi (complex values
//   of the compute precision; empty with the full carrier) in frequency order:
//   the kz = nz/2 plane [S][kx][ky], the ky = ny/2 plane [S][kx][kz < nz/2],
//   the kx = nx/2 plane [S][ky][kz < nz/2], each index the FFT index of its
//   axis (format 1 stored the device's transform-slot order instead).
//
// Reading checks the magic, version, header checksum, payload size and
// payload checksum before anything is returned, so a truncated or altered
// file is refused (PFDD_EINVAL) and the caller's buffers stay untouched.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "pfdd_b200.h"

namespace {

constexpr char kMagic[8] = {'P', 'F', 'D', 'D', 'C', 'K', 'P', '1'};
constexpr uint32_t kVersion = 2, kHeaderBytes = 256;

uint64_t fnv1a(const void *p, size_t n, uint64_t h = 1469598103934665603ull) {
  const unsigned char *b = static_cast<const unsigned char *>(p);
  for (size_t i = 0; i < n; ++i) {
    h ^= b[i];
    h *= 1099511628211ull;
  }
  return h;
}

struct Raw {
  unsigned char b[kHeaderBytes];
  template <typename T> void put(size_t off, T v) { memcpy(b + off, &v, sizeof v); }
  template <typename T> T get(size_t off) const {
    T v;
    memcpy(&v, b + off, sizeof v);
    return v;
  }
};

bool little_endian() {
  const uint16_t x = 1;
  unsigned char c;
  memcpy(&c, &x, 1);
  return c == 1;
}

}  // namespace

extern "C" {

pfdd_status pfdd_checkpoint_write(const char *path, const pfdd_checkpoint_info *info, const void *fields,
                                  const void *carrier) {
  if (!path || !info || (info->field_bytes && !fields) || (info->carrier_bytes && !carrier)) return PFDD_EINVAL;
  if (!little_endian()) return PFDD_EUNSUPPORTED;
  Raw r;
  memset(r.b, 0, sizeof r.b);
  memcpy(r.b, kMagic, 8);
  r.put<uint32_t>(8, kVersion);
  r.put<uint32_t>(12, kHeaderBytes);
  const int32_t ints[8] = {info->nx, info->ny, info->nz, info->n_slip, info->fields, info->precision,
                           info->imag_mode, info->advanced};
  for (int i = 0; i < 8; ++i) r.put<int32_t>(16 + 4 * i, ints[i]);
  r.put<uint64_t>(48, info->field_bytes);
  r.put<uint64_t>(56, info->carrier_bytes);
  for (int i = 0; i < 9; ++i) {
    r.put<double>(64 + 8 * i, info->sigma[i / 3][i % 3]);
    r.put<double>(136 + 8 * i, info->dsigma[i / 3][i % 3]);
  }
  r.put<uint64_t>(208, info->steps);
  uint64_t h = fnv1a(fields, info->field_bytes);
  h = fnv1a(carrier, info->carrier_bytes, h);
  r.put<uint64_t>(216, h);
  r.put<uint64_t>(224, fnv1a(r.b, 224));
  FILE *f = fopen(path, "wb");
  if (!f) return PFDD_EINVAL;
  bool ok = fwrite(r.b, 1, kHeaderBytes, f) == kHeaderBytes;
  ok = ok && fwrite(fields, 1, info->field_bytes, f) == info->field_bytes;
  ok = ok && (!info->carrier_bytes || fwrite(carrier, 1, info->carrier_bytes, f) == info->carrier_bytes);
  ok = (fclose(f) == 0) && ok;
  return ok ? PFDD_OK : PFDD_EINVAL;
}

pfdd_status pfdd_checkpoint_read(const char *path, pfdd_checkpoint_info *info, void *fields, size_t field_cap,
                                 void *carrier, size_t carrier_cap) {
  if (!path || !info) return PFDD_EINVAL;
  if (!little_endian()) return PFDD_EUNSUPPORTED;
  FILE *f = fopen(path, "rb");
  if (!f) return PFDD_EINVAL;
  Raw r;
  if (fread(r.b, 1, kHeaderBytes, f) != kHeaderBytes || memcmp(r.b, kMagic, 8) || r.get<uint32_t>(8) != kVersion ||
      r.get<uint32_t>(12) != kHeaderBytes || r.get<uint64_t>(224) != fnv1a(r.b, 224)) {
    fclose(f);
    return PFDD_EINVAL;
  }
  pfdd_checkpoint_info in;
  memset(&in, 0, sizeof in);
  int32_t ints[8];
  for (int i = 0; i < 8; ++i) ints[i] = r.get<int32_t>(16 + 4 * i);
  in.nx = ints[0]; in.ny = ints[1]; in.nz = ints[2]; in.n_slip = ints[3];
  in.fields = ints[4]; in.precision = ints[5]; in.imag_mode = ints[6]; in.advanced = ints[7];
  in.field_bytes = r.get<uint64_t>(48);
  in.carrier_bytes = r.get<uint64_t>(56);
  for (int i = 0; i < 9; ++i) {
    in.sigma[i / 3][i % 3] = r.get<double>(64 + 8 * i);
    in.dsigma[i / 3][i % 3] = r.get<double>(136 + 8 * i);
  }
  in.steps = r.get<uint64_t>(208);
  if (!fields && !carrier) {   // header only
    fclose(f);
    *info = in;
    return PFDD_OK;
  }
  if (!fields || field_cap < in.field_bytes || (in.carrier_bytes && (!carrier || carrier_cap < in.carrier_bytes))) {
    fclose(f);
    return PFDD_EINVAL;
  }
  // read into scratch first: the caller's buffers change only for a whole, valid file
  std::vector<unsigned char> pay(in.field_bytes + in.carrier_bytes);
  const bool whole = fread(pay.data(), 1, pay.size(), f) == pay.size();
  const bool at_end = whole && fgetc(f) == EOF;
  fclose(f);
  if (!whole || !at_end || fnv1a(pay.data(), pay.size()) != r.get<uint64_t>(216)) return PFDD_EINVAL;
  memcpy(fields, pay.data(), in.field_bytes);
  if (in.carrier_bytes) memcpy(carrier, pay.data() + in.field_bytes, in.carrier_bytes);
  *info = in;
  return PFDD_OK;
}

}  // extern "C"
