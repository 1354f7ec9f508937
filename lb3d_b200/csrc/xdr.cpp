// xdr.cpp -- the reference's XDR files (big-endian IEEE / int32), written
// and read without Sun RPC.  XDR encodes float as 4 and double as 8
// big-endian bytes and int as a 4-byte big-endian two's complement
// (RFC 4506), which is all the reference's xdrf wrapper
// (code/xdrf/libxdrf.m4) emits for checkpoints, topology files, obstacle
// files and dumps.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/lb3dc.h"

namespace {

inline uint64_t bswap64(uint64_t v) { return __builtin_bswap64(v); }
inline uint32_t bswap32(uint32_t v) { return __builtin_bswap32(v); }

void put_d(std::vector<unsigned char> &b, double v) {
  uint64_t u;
  std::memcpy(&u, &v, 8);
  u = bswap64(u);
  const unsigned char *p = reinterpret_cast<const unsigned char *>(&u);
  b.insert(b.end(), p, p + 8);
}
void put_f(std::vector<unsigned char> &b, float v) {
  uint32_t u;
  std::memcpy(&u, &v, 4);
  u = bswap32(u);
  const unsigned char *p = reinterpret_cast<const unsigned char *>(&u);
  b.insert(b.end(), p, p + 4);
}
void put_i(std::vector<unsigned char> &b, int32_t v) {
  uint32_t u = bswap32((uint32_t)v);
  const unsigned char *p = reinterpret_cast<const unsigned char *>(&u);
  b.insert(b.end(), p, p + 4);
}
double get_d(const unsigned char *p) {
  uint64_t u;
  std::memcpy(&u, p, 8);
  u = bswap64(u);
  double v;
  std::memcpy(&v, &u, 8);
  return v;
}
float get_f(const unsigned char *p) {
  uint32_t u;
  std::memcpy(&u, p, 4);
  u = bswap32(u);
  float v;
  std::memcpy(&v, &u, 4);
  return v;
}

bool read_file(const char *path, std::vector<unsigned char> &out) {
  FILE *f = std::fopen(path, "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  long n = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (n < 0) {
    std::fclose(f);
    return false;
  }
  out.resize((size_t)n);
  size_t got = n ? std::fread(out.data(), 1, (size_t)n, f) : 0;
  std::fclose(f);
  return got == (size_t)n;
}

bool write_file(const char *path, const std::vector<unsigned char> &b) {
  FILE *f = std::fopen(path, "wb");
  if (!f) return false;
  size_t put = b.empty() ? 0 : std::fwrite(b.data(), 1, b.size(), f);
  bool ok = (put == b.size());
  ok = (std::fclose(f) == 0) && ok;
  return ok;
}

}  // namespace

extern "C" {

int lb3dc_xdr_read_checkpoint(const char *path, int nx, int ny, int nz, int ncomp, double *n,
                              double *db, double *rock) {
  if (!path || nx < 1 || ny < 1 || nz < 1 || (ncomp != 2 && ncomp != 3) || !n)
    return LB3DC_EINVAL;
  const int nd = ncomp == 3 ? 64 : 39;
  const size_t ns = (size_t)nx * ny * nz;
  std::vector<unsigned char> b;
  if (!read_file(path, b)) return LB3DC_EINVAL;
  if (b.size() != ns * nd * 8) return LB3DC_EINVAL;
  const unsigned char *p = b.data();
  // sites x outermost, then y, then z (code/lb3d_io_checkpoint.F90:842-871)
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z) {
        size_t i = (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z);
        for (int c = 0; c < ncomp; ++c)
          for (int q = 0; q < 19; ++q, p += 8) n[((size_t)c * 19 + q) * ns + i] = get_d(p);
        if (ncomp == 3) {
          p += 3 * 8;  // da: recomputed by every advection step
          for (int k = 0; k < 3; ++k, p += 8)
            if (db) db[(size_t)k * ns + i] = get_d(p);
        }
        if (rock) rock[i] = get_d(p);
        p += 8;
      }
  return LB3DC_OK;
}

int lb3dc_xdr_write_checkpoint(const char *path, int nx, int ny, int nz, int ncomp,
                               const double *n, const double *da, const double *db,
                               const double *rock) {
  if (!path || nx < 1 || ny < 1 || nz < 1 || (ncomp != 2 && ncomp != 3) || !n)
    return LB3DC_EINVAL;
  const size_t ns = (size_t)nx * ny * nz;
  std::vector<unsigned char> b;
  b.reserve(ns * (ncomp == 3 ? 64 : 39) * 8);
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z) {
        size_t i = (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z);
        for (int c = 0; c < ncomp; ++c)
          for (int q = 0; q < 19; ++q) put_d(b, n[((size_t)c * 19 + q) * ns + i]);
        if (ncomp == 3) {
          for (int k = 0; k < 3; ++k) put_d(b, da ? da[(size_t)k * ns + i] : 0.0);
          for (int k = 0; k < 3; ++k) put_d(b, db ? db[(size_t)k * ns + i] : 0.0);
        }
        put_d(b, rock ? rock[i] : 0.0);
      }
  return write_file(path, b) ? LB3DC_OK : LB3DC_EINVAL;
}

int lb3dc_xdr_read_topo(const char *path, double *shear_sum) {
  std::vector<unsigned char> b;
  if (!path || !read_file(path, b) || b.size() < 12) return LB3DC_EINVAL;
  // cdims(3), then 3 ints per rank, then shear_sum (optional)
  size_t nprocs = 1;
  for (int k = 0; k < 3; ++k) {
    uint32_t u;
    std::memcpy(&u, b.data() + 4 * k, 4);
    nprocs *= (size_t)bswap32(u);
  }
  size_t off = 12 + 12 * nprocs;
  if (shear_sum) *shear_sum = (b.size() >= off + 8) ? get_d(b.data() + off) : 0.0;
  return LB3DC_OK;
}

int lb3dc_xdr_write_topo(const char *path, double shear_sum) {
  std::vector<unsigned char> b;
  for (int k = 0; k < 3; ++k) put_i(b, 1);
  for (int k = 0; k < 3; ++k) put_i(b, 0);
  put_d(b, shear_sum);
  return (path && write_file(path, b)) ? LB3DC_OK : LB3DC_EINVAL;
}

int lb3dc_xdr_read_rock(const char *path, int nx, int ny, int nz, double *rock) {
  std::vector<unsigned char> b;
  const size_t ns = (size_t)nx * ny * nz;
  if (!path || !rock || !read_file(path, b) || b.size() < ns * 4) return LB3DC_EINVAL;
  for (size_t i = 0; i < ns; ++i) rock[i] = (get_f(b.data() + 4 * i) > 0.0f) ? 1.0 : 0.0;
  return LB3DC_OK;
}

int lb3dc_xdr_write_rock(const char *path, int nx, int ny, int nz, const double *rock) {
  // createRock's convention: 5.0 for rock, 0.0 for fluid
  // (utils/obstacles/createRock.c:943-954).
  std::vector<unsigned char> b;
  const size_t ns = (size_t)nx * ny * nz;
  if (!path || !rock) return LB3DC_EINVAL;
  b.reserve(ns * 4);
  for (size_t i = 0; i < ns; ++i) put_f(b, rock[i] != 0.0 ? 5.0f : 0.0f);
  return write_file(path, b) ? LB3DC_OK : LB3DC_EINVAL;
}

int lb3dc_xdr_write_field(const char *path, const double *v, long long nsites,
                          int values_per_site, int dump_double) {
  if (!path || !v || nsites < 0 || values_per_site < 1) return LB3DC_EINVAL;
  std::vector<unsigned char> b;
  b.reserve((size_t)nsites * values_per_site * (dump_double ? 8 : 4));
  for (long long i = 0; i < nsites * values_per_site; ++i) {
    if (dump_double)
      put_d(b, v[i]);
    else
      put_f(b, (float)v[i]);
  }
  return write_file(path, b) ? LB3DC_OK : LB3DC_EINVAL;
}

}  // extern "C"
