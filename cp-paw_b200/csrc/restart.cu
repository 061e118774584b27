// Restart records of the WAVES object for one wave-function set: the records
// that WAVES$WRITE / WAVES$READ (src/paw_waves2.f90:3058-3165) put into the
// restart file through WAVES_WRITEPSI (:3168-3357) and WAVES_WRITELAMBDA
// (:3920-4040), read back as WAVES_READPSI (:5147-5513) does for a file of
// the same G set.  Sequential unformatted Fortran records: each record is
// framed by its length in bytes as a 4-byte integer before and after, the
// default of gfortran for records below 2 GiB.
//
// For NKPT = 1, NSPIN = 1, NDIM = 1 and a dynamic restart (NWAVE = 2):
//   separator   NREC, ID 'WAVES', NAME 'NONE', VERSION 'AUG1996', NOTES 'NONE'
//               (SEPARATOR_TYPE, src/paw_report.f90:108-115; characters 32,
//               32, 64 and 256 wide, blank padded)
//   record 1    NKPT, NSPIN, RBAS(3,3), NWAVE
//   record 2    'PSI     ', NGG, NDIM, NB, TSUPER (1/0)
//   record 3    XK(3), IGVEC(3,NGG)
//   NWAVE*NBH   PSI(NGG) of PSI0 for every super wave function, then of PSIM
//   record      'LAMBDA  ', NB, NDIM, NSPIN, NLAMBDA
//   NLAMBDA     RLAM0(NB,NB), then RLAMM (when the handle holds it)
// NREC counts the records after the separator (:3222-3238).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "cuwaves_internal.cuh"

namespace cuw {
namespace {

struct Rec {
  std::vector<unsigned char> b;
  template <class T>
  void put(const T& v) {
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
    b.insert(b.end(), p, p + sizeof(T));
  }
  void put_bytes(const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    b.insert(b.end(), c, c + n);
  }
  void put_chars(const char* s, size_t width) {  // blank padded
    const size_t n = std::strlen(s);
    for (size_t i = 0; i < width; ++i) b.push_back(i < n ? (unsigned char)s[i] : (unsigned char)' ');
  }
};

bool write_rec(FILE* f, const Rec& r) {
  const int32_t n = (int32_t)r.b.size();
  return std::fwrite(&n, 4, 1, f) == 1 && (n == 0 || std::fwrite(r.b.data(), 1, r.b.size(), f) == r.b.size()) &&
         std::fwrite(&n, 4, 1, f) == 1;
}

// Reads one record whose length must be `expect` bytes; a record of another
// length is refused before any buffer is sized from the file's marker.
bool read_rec(FILE* f, std::vector<unsigned char>& out, size_t expect) {
  int32_t n = 0, m = 0;
  if (std::fread(&n, 4, 1, f) != 1 || n < 0 || (size_t)n != expect) return false;
  out.resize((size_t)n);
  if (n && std::fread(out.data(), 1, (size_t)n, f) != (size_t)n) return false;
  return std::fread(&m, 4, 1, f) == 1 && m == n;
}

template <class T>
T get(const std::vector<unsigned char>& b, size_t& off) {
  T v;
  std::memcpy(&v, b.data() + off, sizeof(T));
  off += sizeof(T);
  return v;
}

std::string get_chars(const std::vector<unsigned char>& b, size_t& off, size_t width) {
  std::string s(reinterpret_cast<const char*>(b.data() + off), width);
  off += width;
  while (!s.empty() && s.back() == ' ') s.pop_back();
  return s;
}

// real-space lattice vectors from the reciprocal ones: RBAS^T GBAS = 2 pi
void rbas_of(const double* g, double* r) {
  const double det = g[0] * (g[4] * g[8] - g[7] * g[5]) - g[3] * (g[1] * g[8] - g[7] * g[2]) +
                     g[6] * (g[1] * g[5] - g[4] * g[2]);
  // inverse of G (column-major), then R = 2 pi G^-T
  double inv[9];
  inv[0] = (g[4] * g[8] - g[7] * g[5]) / det;
  inv[3] = -(g[3] * g[8] - g[6] * g[5]) / det;
  inv[6] = (g[3] * g[7] - g[6] * g[4]) / det;
  inv[1] = -(g[1] * g[8] - g[7] * g[2]) / det;
  inv[4] = (g[0] * g[8] - g[6] * g[2]) / det;
  inv[7] = -(g[0] * g[7] - g[6] * g[1]) / det;
  inv[2] = (g[1] * g[5] - g[4] * g[2]) / det;
  inv[5] = -(g[0] * g[5] - g[3] * g[2]) / det;
  inv[8] = (g[0] * g[4] - g[3] * g[1]) / det;
  const double tp = 2.0 * M_PI;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r[i + 3 * j] = tp * inv[j + 3 * i];
}

}  // namespace

int restart_write(Handle* h, const char* path, const double* rbas_in) {
  if (!path) return h->fail(CUW_ERR_ARG, "null path");
  if (h->igvec_h.size() != (size_t)3 * h->d.ngl) return h->fail(CUW_ERR_STATE, "G set not loaded");
  const int ngl = h->d.ngl, nb = h->d.nb, nbh = h->d.nbh;
  double rbas[9];
  if (rbas_in) std::memcpy(rbas, rbas_in, sizeof(rbas));
  else rbas_of(h->gbas, rbas);
  // device state: PSI0, PSIM (padded to ldg), RLAM0, RLAMM
  std::vector<double2> psi((size_t)ngl * nbh * 2), lam((size_t)nb * nb * 2);
  for (int w = 0; w < 2; ++w)
    CUW_TRY(cudaMemcpy2DAsync(psi.data() + (size_t)w * ngl * nbh, sizeof(double2) * ngl, w ? h->g.psim : h->g.psi0,
                              sizeof(double2) * h->ldg, sizeof(double2) * ngl, nbh, cudaMemcpyDeviceToHost,
                              h->stream));
  const int nlambda = h->have_rlamm ? 2 : 1;
  CUW_TRY(cudaMemcpyAsync(lam.data(), h->g.rlam0, sizeof(double2) * nb * nb, cudaMemcpyDeviceToHost, h->stream));
  if (nlambda == 2)
    CUW_TRY(cudaMemcpyAsync(lam.data() + (size_t)nb * nb, h->g.rlamm, sizeof(double2) * nb * nb,
                            cudaMemcpyDeviceToHost, h->stream));
  CUW_TRY(cudaStreamSynchronize(h->stream));
  const int nkpt = 1, nspin = 1, nwave = 2, ndim = 1;
  const int32_t nrec = 1 + 2 + nwave * nbh * nspin + 1 + nspin * nlambda;
  FILE* f = std::fopen(path, "wb");
  if (!f) return h->fail(CUW_ERR_ARG, std::string("cannot open ") + path);
  bool ok = true;
  {
    Rec r;
    r.put(nrec);
    r.put_chars("WAVES", 32);
    r.put_chars("NONE", 32);
    r.put_chars("AUG1996", 64);
    r.put_chars("NONE", 256);
    ok = ok && write_rec(f, r);
  }
  {
    Rec r;
    r.put((int32_t)nkpt);
    r.put((int32_t)nspin);
    r.put_bytes(rbas, sizeof(rbas));
    r.put((int32_t)nwave);
    ok = ok && write_rec(f, r);
  }
  {
    Rec r;
    r.put_chars("PSI", 8);
    r.put((int32_t)ngl);
    r.put((int32_t)ndim);
    r.put((int32_t)nb);
    r.put((int32_t)1);  // super wave functions (TINV)
    ok = ok && write_rec(f, r);
  }
  {
    Rec r;
    const double xk[3] = {0.0, 0.0, 0.0};
    r.put_bytes(xk, sizeof(xk));
    r.put_bytes(h->igvec_h.data(), sizeof(int) * h->igvec_h.size());
    ok = ok && write_rec(f, r);
  }
  for (int w = 0; w < nwave && ok; ++w)
    for (int b = 0; b < nbh && ok; ++b) {
      Rec r;
      r.put_bytes(psi.data() + ((size_t)w * nbh + b) * ngl, sizeof(double2) * ngl);
      ok = ok && write_rec(f, r);
    }
  {
    Rec r;
    r.put_chars("LAMBDA", 8);
    r.put((int32_t)nb);
    r.put((int32_t)ndim);
    r.put((int32_t)nspin);
    r.put((int32_t)nlambda);
    ok = ok && write_rec(f, r);
  }
  for (int l = 0; l < nlambda && ok; ++l) {
    Rec r;
    r.put_bytes(lam.data() + (size_t)l * nb * nb, sizeof(double2) * nb * nb);
    ok = ok && write_rec(f, r);
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return h->fail(CUW_ERR_ARG, std::string("error writing ") + path);
  return CUW_OK;
}

int restart_read(Handle* h, const char* path) {
  if (!path) return h->fail(CUW_ERR_ARG, "null path");
  if (h->igvec_h.size() != (size_t)3 * h->d.ngl) return h->fail(CUW_ERR_STATE, "G set not loaded");
  const int ngl = h->d.ngl, nb = h->d.nb, nbh = h->d.nbh;
  FILE* f = std::fopen(path, "rb");
  if (!f) return h->fail(CUW_ERR_ARG, std::string("cannot open ") + path);
  std::vector<unsigned char> b;
  auto bad = [&](const std::string& m) {
    std::fclose(f);
    return h->fail(CUW_ERR_ARG, "restart file " + std::string(path) + ": " + m);
  };
  size_t off = 0;
  if (!read_rec(f, b, 4 + 32 + 32 + 64 + 256)) return bad("no WAVES separator");
  const int32_t nrec = get<int32_t>(b, off);
  if (get_chars(b, off, 32) != "WAVES") return bad("separator is not WAVES");
  if (!read_rec(f, b, 4 + 4 + 72 + 4)) return bad("record 1");
  off = 0;
  const int nkpt = get<int32_t>(b, off), nspin = get<int32_t>(b, off);
  off += 72;
  const int nwave = get<int32_t>(b, off);
  if (nkpt != 1 || nspin != 1) return bad("one k-point and one spin are supported");
  if (nwave != 1 && nwave != 2) return bad("NWAVE");
  if (!read_rec(f, b, 8 + 16)) return bad("PSI header");
  off = 0;
  if (get_chars(b, off, 8) != "PSI") return bad("PSI key");
  const int ngg = get<int32_t>(b, off), ndim = get<int32_t>(b, off), nbf = get<int32_t>(b, off),
            tsuper = get<int32_t>(b, off);
  if (ndim != 1 || tsuper != 1 || nbf != nb) return bad("NDIM, NB or TSUPER differ from the handle");
  // a G-vector count that no record length can hold is refused before anything is sized from it
  if (ngg <= 0 || (size_t)ngg > ((size_t)INT32_MAX - 24) / 12) return bad("NGG");
  if (!read_rec(f, b, 24 + (size_t)12 * ngg)) return bad("G vectors");
  // the file's G vectors onto this G set (WAVES_READPSI maps by G vector)
  std::map<std::tuple<int, int, int>, int> pos;
  for (int i = 0; i < ngl; ++i) pos[{h->igvec_h[3 * i], h->igvec_h[3 * i + 1], h->igvec_h[3 * i + 2]}] = i;
  std::vector<int> map(ngg, -1);
  for (int i = 0; i < ngg; ++i) {
    int v[3];
    std::memcpy(v, b.data() + 24 + (size_t)12 * i, 12);
    auto it = pos.find({v[0], v[1], v[2]});
    if (it != pos.end()) map[i] = it->second;
  }
  // G vectors of this set that the file lacks start from zero, as in
  // WAVES_READPSI (src/paw_waves2.f90:5395-5403)
  std::vector<double2> psi((size_t)ngl * nbh * 2, make_double2(0.0, 0.0));
  for (int w = 0; w < nwave; ++w)
    for (int ib = 0; ib < nbh; ++ib) {
      if (!read_rec(f, b, sizeof(double2) * ngg)) return bad("wave-function record");
      double2* dst = psi.data() + ((size_t)w * nbh + ib) * ngl;
      for (int i = 0; i < ngg; ++i)
        if (map[i] >= 0) std::memcpy(&dst[map[i]], b.data() + sizeof(double2) * i, sizeof(double2));
    }
  if (nwave == 1) std::memcpy(psi.data() + (size_t)ngl * nbh, psi.data(), sizeof(double2) * ngl * nbh);
  if (!read_rec(f, b, 8 + 16)) return bad("LAMBDA header");
  off = 0;
  if (get_chars(b, off, 8) != "LAMBDA") return bad("LAMBDA key");
  const int nbl = get<int32_t>(b, off);
  off += 8;
  const int nlambda = get<int32_t>(b, off);
  if (nbl != nb || nlambda < 0 || nlambda > 4) return bad("LAMBDA sizes");
  std::vector<double2> lam((size_t)nb * nb * 2, make_double2(0.0, 0.0));
  for (int l = 0; l < nlambda; ++l) {
    if (!read_rec(f, b, sizeof(double2) * nb * nb)) return bad("LAMBDA record");
    if (l < 2) std::memcpy(lam.data() + (size_t)l * nb * nb, b.data(), b.size());
  }
  std::fclose(f);
  if (nrec != 1 + 2 + nwave * nbh + 1 + nlambda) return h->fail(CUW_ERR_ARG, "restart file: NREC of the separator");
  for (int w = 0; w < 2; ++w)
    CUW_TRY(cudaMemcpy2DAsync(w ? h->g.psim : h->g.psi0, sizeof(double2) * h->ldg, psi.data() + (size_t)w * ngl * nbh,
                              sizeof(double2) * ngl, sizeof(double2) * ngl, nbh, cudaMemcpyHostToDevice, h->stream));
  CUW_TRY(cudaMemcpyAsync(h->g.rlam0, lam.data(), sizeof(double2) * nb * nb, cudaMemcpyHostToDevice, h->stream));
  if (nlambda >= 2)
    CUW_TRY(cudaMemcpyAsync(h->g.rlamm, lam.data() + (size_t)nb * nb, sizeof(double2) * nb * nb,
                            cudaMemcpyHostToDevice, h->stream));
  CUW_TRY(cudaStreamSynchronize(h->stream));
  h->have_rlamm = nlambda >= 2;
  h->have_hpsi = false;
  h->have_opsi = false;
  return CUW_OK;
}

}  // namespace cuw

extern "C" int cuwaves_write_restart(cuw_handle* hp, const char* path, const double* rbas) {
  if (!hp) return CUW_ERR_ARG;
  return cuw::restart_write(reinterpret_cast<cuw::Handle*>(hp), path, rbas);
}

extern "C" int cuwaves_read_restart(cuw_handle* hp, const char* path) {
  if (!hp) return CUW_ERR_ARG;
  cuw::Handle* h = reinterpret_cast<cuw::Handle*>(hp);
  h->touch();
  // no C++ exception may cross the C ABI: a host allocation that fails while a
  // damaged file is parsed becomes an argument error of this call
  try {
    return cuw::restart_read(h, path);
  } catch (const std::exception& e) {
    return h->fail(CUW_ERR_ARG, std::string("restart file ") + path + ": " + e.what());
  }
}
