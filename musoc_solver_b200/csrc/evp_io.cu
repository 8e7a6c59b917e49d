// EVP influence file: the record that carries the SEVP operator and its
// precomputed influence matrices from PREP to MAIN.
//
// PREP's INITFS writes one Fortran unformatted sequential record to a
// big-endian file (P/prep_GLOBAL.f90:320, opened by
// OPEN_BIGENDIAN_NEW_BIN_FILE at :40):
//     AL, AR, AB, AT, AC   REAL*4 (I2, J2) each
//     RINV, RINV1          REAL*8 (I2, I2, NB0) / (I2, I2, NB1), or the BIR
//                          strip shapes (IBR2, NB0, NBIR) / (IBR2, NB1, NBIR)
//     IE                   INTEGER*4 (NB0)
// MAIN reads it with an extra REAL*4 (I2, J2) plane OAC after AC
// (M/input_GLOBAL.f90:440-443), which PREP does not write.  The reader here
// takes the record length to decide whether OAC is present and reports it.
//
// Framing (gfortran's sequential unformatted files): a record is one or
// more subrecords, each a 4-byte length marker, the data and the marker
// again.  A subrecord holds at most 2147483639 bytes; a negative leading
// marker means that more subrecords follow, a negative trailing marker that
// the subrecord continues an earlier one.  With CONVERT='BIG_ENDIAN' the
// markers and the data are big-endian.  This file is host code only.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace {

constexpr long long kMaxSubrecord = 2147483639LL;

bool host_little_endian() {
  const uint16_t v = 1;
  return *reinterpret_cast<const uint8_t *>(&v) == 1;
}

// Big-endian bytes of n elements of `size` bytes.
void to_big(const void *src, size_t n, size_t size, std::vector<uint8_t> &out) {
  const uint8_t *s = static_cast<const uint8_t *>(src);
  const size_t off = out.size();
  out.resize(off + n * size);
  uint8_t *d = out.data() + off;
  if (!host_little_endian()) {
    std::memcpy(d, s, n * size);
    return;
  }
  for (size_t k = 0; k < n; ++k)
    for (size_t b = 0; b < size; ++b) d[k * size + b] = s[k * size + size - 1 - b];
}
void from_big(const uint8_t *src, size_t n, size_t size, void *dst) {
  uint8_t *d = static_cast<uint8_t *>(dst);
  if (!host_little_endian()) {
    std::memcpy(d, src, n * size);
    return;
  }
  for (size_t k = 0; k < n; ++k)
    for (size_t b = 0; b < size; ++b) d[k * size + b] = src[k * size + size - 1 - b];
}

bool put_marker(FILE *f, int32_t v) {
  uint8_t b[4];
  from_big(reinterpret_cast<const uint8_t *>(&v), 1, 4, b);  // byte swap is symmetric
  return std::fwrite(b, 1, 4, f) == 4;
}
bool get_marker(FILE *f, int32_t *v) {
  uint8_t b[4];
  if (std::fread(b, 1, 4, f) != 4) return false;
  from_big(b, 1, 4, v);
  return true;
}

int write_record(const char *path, const std::vector<uint8_t> &data, long long max_sub) {
  FILE *f = std::fopen(path, "wb");
  if (!f) return SEVP_BAD_ARG;
  const long long n = (long long)data.size();
  long long pos = 0;
  bool ok = true;
  do {
    const long long len = std::min(max_sub, n - pos);
    const bool more = pos + len < n, cont = pos > 0;
    ok = ok && put_marker(f, (int32_t)(more ? -len : len));
    ok = ok && (len == 0 || std::fwrite(data.data() + pos, 1, (size_t)len, f) == (size_t)len);
    ok = ok && put_marker(f, (int32_t)(cont ? -len : len));
    pos += len;
  } while (ok && pos < n);
  ok = (std::fclose(f) == 0) && ok;
  return ok ? SEVP_OK : SEVP_BAD_ARG;
}

// Reads the first record of the file (all its subrecords).
int read_record(const char *path, std::vector<uint8_t> &data) {
  FILE *f = std::fopen(path, "rb");
  if (!f) return SEVP_BAD_ARG;
  data.clear();
  bool ok = true, first = true;
  for (;;) {
    int32_t lead = 0, trail = 0;
    if (!get_marker(f, &lead)) {
      ok = false;
      break;
    }
    const long long len = lead < 0 ? -(long long)lead : (long long)lead;
    const size_t off = data.size();
    data.resize(off + (size_t)len);
    if (len && std::fread(data.data() + off, 1, (size_t)len, f) != (size_t)len) {
      ok = false;
      break;
    }
    if (!get_marker(f, &trail)) {
      ok = false;
      break;
    }
    const long long tlen = trail < 0 ? -(long long)trail : (long long)trail;
    // markers must agree in length; the trailing sign says "continuation"
    if (tlen != len || (trail < 0) == first) {
      ok = false;
      break;
    }
    first = false;
    if (lead >= 0) break;  // last subrecord
  }
  std::fclose(f);
  return ok ? SEVP_OK : SEVP_BAD_ARG;
}

}  // namespace

extern "C" {

int sevp_evp_write_sub(const char *path, int i2, int j2, const float *al, const float *ar,
                       const float *ab, const float *at, const float *ac, const float *oac,
                       const double *rinv, long long n_rinv, const double *rinv1, long long n_rinv1,
                       const int *ie, int nb0, long long max_subrecord) {
  if (!path || i2 < 1 || j2 < 1 || !al || !ar || !ab || !at || !ac || n_rinv < 0 || n_rinv1 < 0 ||
      (n_rinv && !rinv) || (n_rinv1 && !rinv1) || nb0 < 0 || (nb0 && !ie) || max_subrecord < 1 ||
      max_subrecord > kMaxSubrecord)
    return SEVP_BAD_ARG;
  const size_t plane = (size_t)i2 * j2;
  std::vector<uint8_t> d;
  d.reserve(plane * 4 * 6 + (size_t)(n_rinv + n_rinv1) * 8 + (size_t)nb0 * 4);
  for (const float *a : {al, ar, ab, at, ac}) to_big(a, plane, 4, d);
  if (oac) to_big(oac, plane, 4, d);
  to_big(rinv, (size_t)n_rinv, 8, d);
  to_big(rinv1, (size_t)n_rinv1, 8, d);
  to_big(ie, (size_t)nb0, 4, d);
  return write_record(path, d, max_subrecord);
}

int sevp_evp_write(const char *path, int i2, int j2, const float *al, const float *ar,
                   const float *ab, const float *at, const float *ac, const float *oac,
                   const double *rinv, long long n_rinv, const double *rinv1, long long n_rinv1,
                   const int *ie, int nb0) {
  return sevp_evp_write_sub(path, i2, j2, al, ar, ab, at, ac, oac, rinv, n_rinv, rinv1, n_rinv1,
                            ie, nb0, kMaxSubrecord);
}

int sevp_evp_read(const char *path, int i2, int j2, float *al, float *ar, float *ab, float *at,
                  float *ac, float *oac, double *rinv, long long n_rinv, double *rinv1,
                  long long n_rinv1, int *ie, int nb0, int *has_oac) {
  if (!path || i2 < 1 || j2 < 1 || !al || !ar || !ab || !at || !ac || n_rinv < 0 || n_rinv1 < 0 ||
      (n_rinv && !rinv) || (n_rinv1 && !rinv1) || nb0 < 0 || (nb0 && !ie))
    return SEVP_BAD_ARG;
  std::vector<uint8_t> d;
  int s = read_record(path, d);
  if (s) return s;
  const size_t plane = (size_t)i2 * j2;
  const size_t base = plane * 4 * 5 + (size_t)(n_rinv + n_rinv1) * 8 + (size_t)nb0 * 4;
  int with_oac;
  if (d.size() == base)
    with_oac = 0;
  else if (d.size() == base + plane * 4)
    with_oac = 1;
  else
    return SEVP_BAD_ARG;  // shapes do not match the record
  const uint8_t *p = d.data();
  for (float *a : {al, ar, ab, at, ac}) {
    from_big(p, plane, 4, a);
    p += plane * 4;
  }
  if (with_oac) {
    if (oac) from_big(p, plane, 4, oac);
    p += plane * 4;
  }
  from_big(p, (size_t)n_rinv, 8, rinv);
  p += (size_t)n_rinv * 8;
  from_big(p, (size_t)n_rinv1, 8, rinv1);
  p += (size_t)n_rinv1 * 8;
  from_big(p, (size_t)nb0, 4, ie);
  if (has_oac) *has_oac = with_oac;
  return SEVP_OK;
}

}  // extern "C"
