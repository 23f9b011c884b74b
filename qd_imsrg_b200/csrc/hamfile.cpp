// hamfile.cpp -- the reference's on-disk Hamiltonian format
// (export_hamiltonian / import_hamiltonian, src/ME_general.f90:207-361).
//
// The reference writes a Fortran unformatted sequential file with one record
// per value: every FP64 entry is framed by 4-byte record markers holding 8
// (gfortran's and ifort's default), 16 bytes per entry, no header.  The order
// is the loop order of export_hamiltonian:
//   E0; fhh(i,j) i=1..n, j=1..n (row by row); fph(i,j) i=1..m-n, j=1..n;
//   fpp(i,j) i,j=1..m-n; then per block q = 1..nblock: Vhhhh(i,j), Vpppp,
//   Vpphh (i over pp, j over hh), Vphph, Vphhh (i over ph, j over hh), Vppph
//   (i over pp, j over ph), each row by row.
// Note the part order differs from vectorize (fph before fpp, Vphhh before
// Vppph) and every matrix is written row by row, so the file is a
// permutation of the vectorize array.  The reference prefixes the name with
// '../hamiltonians/'; here the caller passes the full path.
#include <cstdio>
#include <cstring>
#include <vector>

#include "qd_internal.hpp"

namespace qd {
namespace {

// vectorize index of the k-th value in file order, k = 0..neq-1
template <class F>
void file_order(const qd_layout* L, F&& visit) {
  const int n = L->n, mp = L->mp;
  visit((i64)0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) visit(L->o_fhh + i + (i64)j * n);
  for (int i = 0; i < mp; ++i)
    for (int j = 0; j < n; ++j) visit(L->o_fph + i + (i64)j * mp);
  for (int i = 0; i < mp; ++i)
    for (int j = 0; j < mp; ++j) visit(L->o_fpp + i + (i64)j * mp);
  for (int q = 0; q < L->nblock; ++q) {
    const int nh = L->blk[q].x, nb = L->blk[q].y, np = L->blk[q].z;
    const i64* o = &L->boff[6 * q];
    auto mat = [&](i64 off, int rows, int cols) {
      for (int i = 0; i < rows; ++i)
        for (int j = 0; j < cols; ++j) visit(off + i + (i64)j * rows);
    };
    mat(o[0], nh, nh);  // Vhhhh
    mat(o[1], np, np);  // Vpppp
    mat(o[2], np, nh);  // Vpphh
    mat(o[3], nb, nb);  // Vphph
    mat(o[5], nb, nh);  // Vphhh
    mat(o[4], np, nb);  // Vppph
  }
}

constexpr size_t CHUNK = 1 << 16;  // entries per buffered write / read

}  // namespace
}  // namespace qd

using namespace qd;

extern "C" {

int qd_hamiltonian_write(const qd_layout* L, const double* vec, const char* path) {
  if (!L || !vec || !path) {
    set_error("qd_hamiltonian_write: null argument");
    return QD_ERR_ARG;
  }
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    set_error("qd_hamiltonian_write: cannot open %s for writing", path);
    return QD_ERR_ARG;
  }
  std::vector<unsigned char> buf;
  buf.reserve(CHUNK * 16);
  const int marker = 8;
  bool ok = true;
  file_order(L, [&](i64 idx) {
    unsigned char rec[16];
    std::memcpy(rec, &marker, 4);
    std::memcpy(rec + 4, vec + idx, 8);
    std::memcpy(rec + 12, &marker, 4);
    buf.insert(buf.end(), rec, rec + 16);
    if (buf.size() >= CHUNK * 16) {
      ok = ok && std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
      buf.clear();
    }
  });
  if (!buf.empty()) ok = ok && std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) {
    set_error("qd_hamiltonian_write: write to %s failed", path);
    return QD_ERR_ARG;
  }
  return QD_OK;
}

int qd_hamiltonian_read(const qd_layout* L, double* vec, const char* path) {
  if (!L || !vec || !path) {
    set_error("qd_hamiltonian_read: null argument");
    return QD_ERR_ARG;
  }
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_error("qd_hamiltonian_read: cannot open %s", path);
    return QD_ERR_ARG;
  }
  std::fseek(f, 0, SEEK_END);
  const long long size = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (size != 16LL * L->neq) {
    std::fclose(f);
    set_error("qd_hamiltonian_read: %s holds %lld bytes, the layout needs %lld (16 per entry)", path, size,
              16LL * (long long)L->neq);
    return QD_ERR_ARG;
  }
  std::vector<unsigned char> buf(CHUNK * 16);
  size_t have = 0, pos = 0;
  bool ok = true;
  file_order(L, [&](i64 idx) {
    if (!ok) return;
    if (pos == have) {
      have = std::fread(buf.data(), 1, buf.size(), f);
      pos = 0;
      if (have < 16) {
        ok = false;
        return;
      }
    }
    int m1, m2;
    std::memcpy(&m1, &buf[pos], 4);
    std::memcpy(vec + idx, &buf[pos + 4], 8);
    std::memcpy(&m2, &buf[pos + 12], 4);
    ok = m1 == 8 && m2 == 8;
    pos += 16;
  });
  std::fclose(f);
  if (!ok) {
    set_error("qd_hamiltonian_read: %s is not a file of 8-byte records", path);
    return QD_ERR_ARG;
  }
  return QD_OK;
}

int qd_export_hamiltonian(const qd_op* H, const char* path) {
  if (!H) {
    set_error("qd_export_hamiltonian: null operator");
    return QD_ERR_ARG;
  }
  std::vector<double> v((size_t)H->L->neq);
  int rc = qd_op_download(H, v.data(), H->L->neq);
  if (rc) return rc;
  return qd_hamiltonian_write(H->L, v.data(), path);
}

int qd_import_hamiltonian(qd_op* H, const char* path) {
  if (!H) {
    set_error("qd_import_hamiltonian: null operator");
    return QD_ERR_ARG;
  }
  std::vector<double> v((size_t)H->L->neq);
  int rc = qd_hamiltonian_read(H->L, v.data(), path);
  if (rc) return rc;
  return qd_op_upload(H, v.data(), H->L->neq);
}

}  // extern "C"
