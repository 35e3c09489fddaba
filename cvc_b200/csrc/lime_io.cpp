// LIME / SciDAC / ILDG file I/O for gauge fields, propagators and contractions,
// on the host.  The reference does this with the c-lime (or lemon) library in
// io.c, gauge_io.c, propagator_io.c and contractions_io.c; this file writes and
// reads the same files with its own implementation of the published formats:
//
//  * LIME record: a 144-byte header -- magic 0x456789ab (4 bytes), version 1
//    (2 bytes), flags (2 bytes; bit 15 message begin MB, bit 14 message end
//    ME), data length (8 bytes), type string (128 bytes, NUL padded), all
//    integers big-endian -- then the data, zero-padded to a multiple of 8.
//  * Binary records hold big-endian IEEE numbers, 64 or 32 bit (the reader
//    takes the precision from the record length).
//  * SciDAC checksum (dml.c:22-50): per site, the CRC-32 (zlib polynomial) of
//    the site's bytes as stored in the file, rotated left by rank % 29 (suma)
//    and rank % 31 (sumb), XORed over all sites.
//
// Site order in the files: gauge and propagator records run t, z, y, x with
// x fastest (io.c:282-285, propagator_io.c:363-366), rank = ((t LZ + z) LY +
// y) LX + x; ILDG links come in the order x, y, z, t of the direction (io.c:
// 299-322).  Contraction records run t, x, y, z with z fastest (CVC's own
// order, contractions_io.c:102-106).  Fields in memory are CVC's layouts.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "cvcb_internal.h"

namespace {

// ---- CRC-32 (reflected, polynomial 0xEDB88320) and the SciDAC checksum ------
uint32_t g_crc_table[256];
std::once_flag g_crc_once;

void crc_init() {
  for (uint32_t n = 0; n < 256; ++n) {
    uint32_t c = n;
    for (int k = 0; k < 8; ++k) c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
    g_crc_table[n] = c;
  }
}

uint32_t crc32_update(uint32_t crc, const unsigned char *p, size_t n) {
  std::call_once(g_crc_once, crc_init);
  crc = ~crc;
  while (n--) crc = g_crc_table[(crc ^ *p++) & 0xffu] ^ (crc >> 8);
  return ~crc;
}

uint32_t rotl32(uint32_t w, unsigned r) { return r ? (w << r) | (w >> (32 - r)) : w; }

struct Checksum {
  uint32_t a = 0, b = 0;
  void accum(uint64_t rank, const void *buf, size_t n) {
    const uint32_t w = crc32_update(0, static_cast<const unsigned char *>(buf), n);
    const uint32_t r = (uint32_t)rank;  // DML_SiteRank is 32 bits wide (dml.h:17)
    a ^= rotl32(w, r % 29);
    b ^= rotl32(w, r % 31);
  }
};

// ---- big-endian helpers -----------------------------------------------------
void put_be(unsigned char *p, uint64_t v, int n) {
  for (int i = n - 1; i >= 0; --i) {
    p[i] = (unsigned char)(v & 0xff);
    v >>= 8;
  }
}
uint64_t get_be(const unsigned char *p, int n) {
  uint64_t v = 0;
  for (int i = 0; i < n; ++i) v = (v << 8) | p[i];
  return v;
}
// n reals -> big-endian bytes in `out` (8 n or 4 n bytes)
void reals_to_be(unsigned char *out, const double *v, int n, int prec) {
  for (int i = 0; i < n; ++i) {
    if (prec == 32) {
      const float f = (float)v[i];
      uint32_t u;
      std::memcpy(&u, &f, 4);
      put_be(out + 4 * i, u, 4);
    } else {
      uint64_t u;
      std::memcpy(&u, &v[i], 8);
      put_be(out + 8 * i, u, 8);
    }
  }
}
void be_to_reals(double *v, const unsigned char *in, int n, int prec) {
  for (int i = 0; i < n; ++i) {
    if (prec == 32) {
      const uint32_t u = (uint32_t)get_be(in + 4 * i, 4);
      float f;
      std::memcpy(&f, &u, 4);
      v[i] = f;
    } else {
      const uint64_t u = get_be(in + 8 * i, 8);
      std::memcpy(&v[i], &u, 8);
    }
  }
}

// ---- LIME records -------------------------------------------------------------
constexpr uint32_t kLimeMagic = 0x456789abu;
constexpr int kLimeHeader = 144;

struct File {
  FILE *f = nullptr;
  File(const char *name, const char *mode) : f(std::fopen(name, mode)) {}
  ~File() {
    if (f) std::fclose(f);
  }
};

int write_header(FILE *f, const char *type, uint64_t bytes, bool mb, bool me) {
  unsigned char h[kLimeHeader] = {0};
  put_be(h, kLimeMagic, 4);
  put_be(h + 4, 1, 2);
  put_be(h + 6, (mb ? 0x8000u : 0) | (me ? 0x4000u : 0), 2);
  put_be(h + 8, bytes, 8);
  std::strncpy(reinterpret_cast<char *>(h + 16), type, 127);
  return std::fwrite(h, 1, kLimeHeader, f) == (size_t)kLimeHeader ? 0 : -1;
}
int write_pad(FILE *f, uint64_t bytes) {
  static const unsigned char zero[8] = {0};
  const size_t pad = (size_t)((8 - bytes % 8) % 8);
  return std::fwrite(zero, 1, pad, f) == pad ? 0 : -1;
}
int write_record(FILE *f, const char *type, const void *data, uint64_t bytes, bool mb, bool me) {
  if (write_header(f, type, bytes, mb, me)) return -1;
  if (bytes && std::fwrite(data, 1, (size_t)bytes, f) != (size_t)bytes) return -1;
  return write_pad(f, bytes);
}

struct Record {
  std::string type;
  uint64_t bytes;
  long offset;  // of the data
};

// All record headers of a LIME file; false on a malformed header.
bool scan(FILE *f, std::vector<Record> &out) {
  std::fseek(f, 0, SEEK_SET);
  unsigned char h[kLimeHeader];
  while (true) {
    const size_t got = std::fread(h, 1, kLimeHeader, f);
    if (got == 0) return true;
    if (got != (size_t)kLimeHeader || get_be(h, 4) != kLimeMagic) return false;
    Record r;
    r.bytes = get_be(h + 8, 8);
    char type[129];
    std::memcpy(type, h + 16, 128);
    type[128] = 0;
    r.type = type;
    r.offset = std::ftell(f);
    out.push_back(r);
    const uint64_t padded = (r.bytes + 7) / 8 * 8;
    if (std::fseek(f, (long)padded, SEEK_CUR)) return false;
  }
}

// The position-th record of the given type (0-based), or nullptr.
const Record *find(const std::vector<Record> &recs, const char *type, int position) {
  int k = -1;
  for (const Record &r : recs)
    if (r.type == type && ++k == position) return &r;
  return nullptr;
}

std::string checksum_xml(const Checksum &c) {
  char buf[256];
  std::snprintf(buf, sizeof buf,
                "<?xml version=\"1.0\" encoding=\"UTF-8\"?><scidacChecksum><version>1.0</version>"
                "<suma>%#010x</suma><sumb>%#010x</sumb></scidacChecksum>",
                c.a, c.b);
  return buf;
}

bool dims_ok(int T, int LX, int LY, int LZ) { return T > 0 && LX > 0 && LY > 0 && LZ > 0; }

size_t lex(int t, int x, int y, int z, int LX, int LY, int LZ) {
  return (((size_t)t * LX + x) * LY + y) * LZ + z;
}

void put_sums(uint32_t *out, const Checksum &c) {
  if (out) {
    out[0] = c.a;
    out[1] = c.b;
  }
}

}  // namespace

extern "C" {

int cvcb_crc32(uint32_t crc, const void *buf, size_t len, uint32_t *out) {
  if ((!buf && len) || !out) return CVCB_ERR_NULL;
  *out = crc32_update(crc, static_cast<const unsigned char *>(buf), len);
  return CVCB_OK;
}

int cvcb_dml_checksum_accum(uint32_t sums[2], uint64_t rank, const void *buf, size_t size) {
  if (!sums || (!buf && size)) return CVCB_ERR_NULL;
  Checksum c;
  c.a = sums[0];
  c.b = sums[1];
  c.accum(rank, buf, size);
  sums[0] = c.a;
  sums[1] = c.b;
  return CVCB_OK;
}

// ---- gauge fields (ILDG) ----------------------------------------------------
int cvcb_read_lime_gauge_field_doubleprec(const char *filename, double *gauge, int T, int LX,
                                          int LY, int LZ, uint32_t checksum[2]) {
  if (!filename || !gauge) return CVCB_ERR_NULL;
  if (!dims_ok(T, LX, LY, LZ)) return CVCB_ERR_ARG;
  File in(filename, "rb");
  if (!in.f) {
    cvcb::set_error("cannot open %s", filename);
    return CVCB_ERR_ARG;
  }
  std::vector<Record> recs;
  if (!scan(in.f, recs)) {
    cvcb::set_error("%s is not a LIME file", filename);
    return CVCB_ERR_ARG;
  }
  const Record *r = find(recs, "ildg-binary-data", 0);
  if (!r) {
    cvcb::set_error("no ildg-binary-data record in %s", filename);
    return CVCB_ERR_ARG;
  }
  const uint64_t V = (uint64_t)T * LX * LY * LZ;
  int prec;
  if (r->bytes == V * 72 * 8) prec = 64;
  else if (r->bytes == V * 72 * 4) prec = 32;  // io.c:254-268: falls back to single precision
  else {
    cvcb::set_error("ildg-binary-data of %llu bytes does not fit the lattice",
                    (unsigned long long)r->bytes);
    return CVCB_ERR_ARG;
  }
  const size_t site_bytes = (size_t)72 * (prec / 8);
  std::vector<unsigned char> buf(site_bytes * LX);
  std::fseek(in.f, r->offset, SEEK_SET);
  Checksum cs;
  double v[72];
  for (int t = 0; t < T; ++t)
    for (int z = 0; z < LZ; ++z)
      for (int y = 0; y < LY; ++y) {
        if (std::fread(buf.data(), 1, buf.size(), in.f) != buf.size()) {
          cvcb::set_error("short read in %s", filename);
          return CVCB_ERR_ARG;
        }
        for (int x = 0; x < LX; ++x) {
          const unsigned char *site = buf.data() + site_bytes * x;
          cs.accum((((uint64_t)t * LZ + z) * LY + y) * LX + x, site, site_bytes);
          be_to_reals(v, site, 72, prec);
          double *g = gauge + 72 * lex(t, x, y, z, LX, LY, LZ);
          // file direction order x, y, z, t -> CVC t, x, y, z
          std::memcpy(g + 18, v, 54 * sizeof(double));
          std::memcpy(g, v + 54, 18 * sizeof(double));
        }
      }
  put_sums(checksum, cs);
  return CVCB_OK;
}

int cvcb_write_lime_gauge_field(const char *filename, const double *gauge, int T, int LX, int LY,
                                int LZ, int prec, uint32_t checksum[2]) {
  if (!filename || !gauge) return CVCB_ERR_NULL;
  if (!dims_ok(T, LX, LY, LZ) || (prec != 32 && prec != 64)) return CVCB_ERR_ARG;
  File out(filename, "wb");
  if (!out.f) {
    cvcb::set_error("cannot create %s", filename);
    return CVCB_ERR_ARG;
  }
  char fmt[1024];
  std::snprintf(fmt, sizeof fmt,
                "<?xml version=\"1.0\" encoding=\"UTF-8\"?>\n"
                "<ildgFormat xmlns=\"http://www.lqcd.org/ildg\"\n"
                "            xmlns:xsi=\"http://www.w3.org/2001/XMLSchema-instance\"\n"
                "            xsi:schemaLocation=\"http://www.lqcd.org/ildg filefmt.xsd\">\n"
                "  <version> 1.0 </version>\n  <field> su3gauge </field>\n"
                "  <precision> %d </precision>\n  <lx> %d </lx>\n  <ly> %d </ly>\n"
                "  <lz> %d </lz>\n  <lt> %d </lt>\n</ildgFormat>",
                prec, LX, LY, LZ, T);
  if (write_record(out.f, "ildg-format", fmt, std::strlen(fmt), true, false)) return CVCB_ERR_ARG;
  const uint64_t V = (uint64_t)T * LX * LY * LZ;
  const size_t site_bytes = (size_t)72 * (prec / 8);
  const uint64_t bytes = V * site_bytes;
  if (write_header(out.f, "ildg-binary-data", bytes, false, false)) return CVCB_ERR_ARG;
  std::vector<unsigned char> buf(site_bytes * LX);
  Checksum cs;
  double v[72];
  for (int t = 0; t < T; ++t)
    for (int z = 0; z < LZ; ++z)
      for (int y = 0; y < LY; ++y) {
        for (int x = 0; x < LX; ++x) {
          const double *g = gauge + 72 * lex(t, x, y, z, LX, LY, LZ);
          std::memcpy(v, g + 18, 54 * sizeof(double));
          std::memcpy(v + 54, g, 18 * sizeof(double));
          unsigned char *site = buf.data() + site_bytes * x;
          reals_to_be(site, v, 72, prec);
          cs.accum((((uint64_t)t * LZ + z) * LY + y) * LX + x, site, site_bytes);
        }
        if (std::fwrite(buf.data(), 1, buf.size(), out.f) != buf.size()) return CVCB_ERR_ARG;
      }
  if (write_pad(out.f, bytes)) return CVCB_ERR_ARG;
  const std::string ck = checksum_xml(cs);
  if (write_record(out.f, "scidac-checksum", ck.data(), ck.size(), false, true)) return CVCB_ERR_ARG;
  put_sums(checksum, cs);
  return CVCB_OK;
}

// ---- propagators (SciDAC Dirac fermion fields) --------------------------------
int cvcb_read_lime_spinor(double *s, const char *filename, int position, int T, int LX, int LY,
                          int LZ, uint32_t checksum[2]) {
  if (!s || !filename) return CVCB_ERR_NULL;
  if (!dims_ok(T, LX, LY, LZ) || position < 0) return CVCB_ERR_ARG;
  File in(filename, "rb");
  if (!in.f) {
    cvcb::set_error("cannot open %s", filename);
    return CVCB_ERR_ARG;
  }
  std::vector<Record> recs;
  if (!scan(in.f, recs)) {
    cvcb::set_error("%s is not a LIME file", filename);
    return CVCB_ERR_ARG;
  }
  const Record *r = find(recs, "scidac-binary-data", position);
  if (!r) {
    cvcb::set_error("no scidac-binary-data record %d in %s", position, filename);
    return CVCB_ERR_ARG;
  }
  const uint64_t V = (uint64_t)T * LX * LY * LZ;
  int prec;
  if (r->bytes == V * 24 * 8) prec = 64;
  else if (r->bytes == V * 24 * 4) prec = 32;
  else {
    cvcb::set_error("scidac-binary-data of %llu bytes is not a Dirac field on this lattice",
                    (unsigned long long)r->bytes);
    return CVCB_ERR_ARG;
  }
  const size_t site_bytes = (size_t)24 * (prec / 8);
  std::vector<unsigned char> buf(site_bytes * LX);
  std::fseek(in.f, r->offset, SEEK_SET);
  Checksum cs;
  for (int t = 0; t < T; ++t)
    for (int z = 0; z < LZ; ++z)
      for (int y = 0; y < LY; ++y) {
        if (std::fread(buf.data(), 1, buf.size(), in.f) != buf.size()) {
          cvcb::set_error("short read in %s", filename);
          return CVCB_ERR_ARG;
        }
        for (int x = 0; x < LX; ++x) {
          const unsigned char *site = buf.data() + site_bytes * x;
          cs.accum((((uint64_t)t * LZ + z) * LY + y) * LX + x, site, site_bytes);
          be_to_reals(s + 24 * lex(t, x, y, z, LX, LY, LZ), site, 24, prec);
        }
      }
  put_sums(checksum, cs);
  return CVCB_OK;
}

namespace {
int append_spinor(FILE *f, const double *s, int prec, int T, int LX, int LY, int LZ, Checksum &cs) {
  const uint64_t V = (uint64_t)T * LX * LY * LZ;
  const size_t site_bytes = (size_t)24 * (prec / 8);
  const uint64_t bytes = V * site_bytes;
  if (write_header(f, "scidac-binary-data", bytes, false, true)) return -1;
  std::vector<unsigned char> buf(site_bytes * LX);
  for (int t = 0; t < T; ++t)
    for (int z = 0; z < LZ; ++z)
      for (int y = 0; y < LY; ++y) {
        for (int x = 0; x < LX; ++x) {
          unsigned char *site = buf.data() + site_bytes * x;
          reals_to_be(site, s + 24 * lex(t, x, y, z, LX, LY, LZ), 24, prec);
          cs.accum((((uint64_t)t * LZ + z) * LY + y) * LX + x, site, site_bytes);
        }
        if (std::fwrite(buf.data(), 1, buf.size(), f) != buf.size()) return -1;
      }
  if (write_pad(f, bytes)) return -1;
  const std::string ck = checksum_xml(cs);
  return write_record(f, "scidac-checksum", ck.data(), ck.size(), true, false);
}
}  // namespace

int cvcb_write_lime_spinor(const double *s, const char *filename, int append, int prec, int T,
                           int LX, int LY, int LZ, uint32_t checksum[2]) {
  if (!s || !filename) return CVCB_ERR_NULL;
  if (!dims_ok(T, LX, LY, LZ) || (prec != 32 && prec != 64)) return CVCB_ERR_ARG;
  File out(filename, append ? "ab" : "wb");
  if (!out.f) {
    cvcb::set_error("cannot open %s for writing", filename);
    return CVCB_ERR_ARG;
  }
  Checksum cs;
  if (append_spinor(out.f, s, prec, T, LX, LY, LZ, cs)) return CVCB_ERR_ARG;
  put_sums(checksum, cs);
  return CVCB_OK;
}

int cvcb_write_propagator(const double *s, const char *filename, int prec, int T, int LX, int LY,
                          int LZ, uint32_t checksum[2]) {
  if (!s || !filename) return CVCB_ERR_NULL;
  if (!dims_ok(T, LX, LY, LZ) || (prec != 32 && prec != 64)) return CVCB_ERR_ARG;
  File out(filename, "wb");
  if (!out.f) {
    cvcb::set_error("cannot create %s", filename);
    return CVCB_ERR_ARG;
  }
  char fmt[512];
  std::snprintf(fmt, sizeof fmt,
                "<?xml version=\"1.0\" encoding=\"UTF-8\"?>\n<etmcFormat>\n"
                "<field>diracFermion</field>\n<precision>%d</precision>\n<flavours>%d</flavours>\n"
                "<lx>%d</lx>\n<ly>%d</ly>\n<lz>%d</lz>\n<lt>%d</lt>\n</etmcFormat>",
                prec, 1, LX, LY, LZ, T);
  if (write_record(out.f, "etmc-propagator-format", fmt, std::strlen(fmt), true, false))
    return CVCB_ERR_ARG;
  Checksum cs;
  if (append_spinor(out.f, s, prec, T, LX, LY, LZ, cs)) return CVCB_ERR_ARG;
  put_sums(checksum, cs);
  return CVCB_OK;
}

// ---- contractions (N complex components per site, CVC site order) ----------
int cvcb_write_lime_contraction(const double *s, const char *filename, int prec, int N,
                                const char *type, int gid, int sid, int T, int LX, int LY, int LZ,
                                uint32_t checksum[2]) {
  if (!s || !filename || !type) return CVCB_ERR_NULL;
  if (!dims_ok(T, LX, LY, LZ) || (prec != 32 && prec != 64) || N <= 0) return CVCB_ERR_ARG;
  File out(filename, "wb");
  if (!out.f) {
    cvcb::set_error("cannot create %s", filename);
    return CVCB_ERR_ARG;
  }
  char fmt[1024];
  std::snprintf(fmt, sizeof fmt,
                "<?xml version=\"1.0\" encoding=\"UTF-8\"?>\n<cvcFormat>\n<type>%s</type>\n"
                "<precision>%d</precision>\n<components>%d</components>\n<lx>%d</lx>\n"
                "<ly>%d</ly>\n<lz>%d</lz>\n<lt>%d</lt>\n<nconf>%d</nconf>\n<source>%d</source>\n"
                "</cvcFormat>",
                type, prec, N, LX, LY, LZ, T, gid, sid);
  if (write_record(out.f, "cvc_contraction-format", fmt, std::strlen(fmt), true, true))
    return CVCB_ERR_ARG;
  const uint64_t V = (uint64_t)T * LX * LY * LZ;
  const size_t site_bytes = (size_t)2 * N * (prec / 8);
  const uint64_t bytes = V * site_bytes;
  if (write_header(out.f, "scidac-binary-data", bytes, true, false)) return CVCB_ERR_ARG;
  std::vector<unsigned char> buf(site_bytes);
  Checksum cs;
  for (uint64_t ix = 0; ix < V; ++ix) {  // t, x, y, z with z fastest = CVC order
    reals_to_be(buf.data(), s + 2 * (size_t)N * ix, 2 * N, prec);
    cs.accum(ix, buf.data(), site_bytes);
    if (std::fwrite(buf.data(), 1, site_bytes, out.f) != site_bytes) return CVCB_ERR_ARG;
  }
  if (write_pad(out.f, bytes)) return CVCB_ERR_ARG;
  char ck[256];
  std::snprintf(ck, sizeof ck,
                "<?xml version=\"1.0\" encoding=\"UTF-8\"?>\n<scidacChecksum>\n  <version>1.0</version>\n"
                "  <suma>%08x</suma>\n  <sumb>%08x</sumb>\n</scidacChecksum>",
                cs.a, cs.b);
  if (write_record(out.f, "scidac-checksum", ck, std::strlen(ck), false, true)) return CVCB_ERR_ARG;
  put_sums(checksum, cs);
  return CVCB_OK;
}

int cvcb_read_lime_contraction(double *s, const char *filename, int N, int position, int T, int LX,
                               int LY, int LZ, uint32_t checksum[2]) {
  if (!s || !filename) return CVCB_ERR_NULL;
  if (!dims_ok(T, LX, LY, LZ) || N <= 0 || position < 0) return CVCB_ERR_ARG;
  File in(filename, "rb");
  if (!in.f) {
    cvcb::set_error("cannot open %s", filename);
    return CVCB_ERR_ARG;
  }
  std::vector<Record> recs;
  if (!scan(in.f, recs)) {
    cvcb::set_error("%s is not a LIME file", filename);
    return CVCB_ERR_ARG;
  }
  const Record *r = find(recs, "scidac-binary-data", position);
  if (!r) {
    cvcb::set_error("no scidac-binary-data record %d in %s", position, filename);
    return CVCB_ERR_ARG;
  }
  const uint64_t V = (uint64_t)T * LX * LY * LZ;
  int prec;
  if (r->bytes == V * 2 * N * 8) prec = 64;
  else if (r->bytes == V * 2 * N * 4) prec = 32;
  else {
    cvcb::set_error("record of %llu bytes does not hold %d components on this lattice",
                    (unsigned long long)r->bytes, N);
    return CVCB_ERR_ARG;
  }
  const size_t site_bytes = (size_t)2 * N * (prec / 8);
  std::vector<unsigned char> buf(site_bytes);
  std::fseek(in.f, r->offset, SEEK_SET);
  Checksum cs;
  for (uint64_t ix = 0; ix < V; ++ix) {
    if (std::fread(buf.data(), 1, site_bytes, in.f) != site_bytes) {
      cvcb::set_error("short read in %s", filename);
      return CVCB_ERR_ARG;
    }
    cs.accum(ix, buf.data(), site_bytes);
    be_to_reals(s + 2 * (size_t)N * ix, buf.data(), 2 * N, prec);
  }
  put_sums(checksum, cs);
  return CVCB_OK;
}

}  // extern "C"
