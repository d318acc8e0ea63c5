// fortran_io.cu -- the reference's field output and restart files
// (nse_dominik.f:2606-2793: OUTPUT, OUTFIELD, READFIELD) in the byte layout
// gfortran gives them, so a run of this library and a run of the reference
// can read each other's files.
//
// FORM='UNFORMATTED' sequential files: every WRITE statement is one record,
// framed by its length in bytes as a 4-byte little-endian integer before and
// after the data.  OUTPUT writes one record per interior cell to each .dat
// file (i fastest), three values to velocity.dat; field.u holds one record
// of nine values per padded cell; OUTFIELD's field.u starts with a record
// holding the simulation time.  temperature_check.dat is list-directed
// (formatted) text, written here with gfortran's list-directed layout for
// REAL(8) (a blank, then G25.17E3 editing); that layout is restated from
// gfortran's documented behaviour and is not checked against a gfortran run.
//
// Host code only: the resident entry points (runtime.cu) download the fields
// and call these writers; the legacy entry points take host arrays directly.
#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <sys/stat.h>

#include <string>
#include <vector>

#include "common.cuh"

namespace nse {

namespace {

// buffered writer of gfortran sequential unformatted records
struct RecWriter {
  FILE* f = nullptr;
  std::vector<char> buf;
  bool ok = true;
  explicit RecWriter(const std::string& path) {
    f = fopen(path.c_str(), "wb");
    ok = f != nullptr;
    buf.reserve(1 << 22);
  }
  ~RecWriter() { close(); }
  void put(const void* p, size_t n) {
    const char* c = static_cast<const char*>(p);
    buf.insert(buf.end(), c, c + n);
    if (buf.size() >= (1u << 22)) flush();
  }
  void flush() {
    if (f && !buf.empty()) ok = ok && fwrite(buf.data(), 1, buf.size(), f) == buf.size();
    buf.clear();
  }
  // one record of n doubles
  void rec(const double* v, int n) {
    const int32_t len = (int32_t)(n * sizeof(double));
    put(&len, 4);
    put(v, n * sizeof(double));
    put(&len, 4);
  }
  void rec_ints(const int32_t* v, int n) {
    const int32_t len = (int32_t)(n * sizeof(int32_t));
    put(&len, 4);
    put(v, n * sizeof(int32_t));
    put(&len, 4);
  }
  bool close() {
    if (f) {
      flush();
      ok = (fclose(f) == 0) && ok;
      f = nullptr;
    }
    return ok;
  }
};

// sequential reader of the same records
struct RecReader {
  FILE* f = nullptr;
  explicit RecReader(const std::string& path) { f = fopen(path.c_str(), "rb"); }
  ~RecReader() {
    if (f) fclose(f);
  }
  bool rec(double* v, int n) {
    int32_t a = 0, b = 0;
    if (fread(&a, 4, 1, f) != 1 || a != (int32_t)(n * sizeof(double))) return false;
    if (fread(v, sizeof(double), n, f) != (size_t)n) return false;
    if (fread(&b, 4, 1, f) != 1 || b != a) return false;
    return true;
  }
};

bool ensure_dir(const std::string& dir) {
  if (mkdir(dir.c_str(), 0755) == 0 || errno == EEXIST) return true;
  set_error(NSE_ERR_ARG, "cannot create directory %s: %s", dir.c_str(), strerror(errno));
  return false;
}

// one REAL(8) item of list-directed output: a blank, then G25.17E3
void list_item(std::string& line, double v) {
  char num[96], field[160];
  if (v == 0.0 || (fabs(v) >= 0.1 && fabs(v) < 1e17)) {
    int decimals = 16;  // zero: 0.0000000000000000
    if (v != 0.0) {
      // decimal exponent of v rounded to 17 significant digits
      char e[64];
      snprintf(e, sizeof e, "%.16e", v);
      const int ex = atoi(strchr(e, 'e') + 1);
      decimals = 17 - (ex + 1);
      if (ex + 1 > 17 || ex < -1) decimals = -1;  // rounded out of the F range
    }
    if (decimals >= 0) {
      snprintf(num, sizeof num, "%.*f", decimals, v);
      snprintf(field, sizeof field, "%20s     ", num);  // the exponent field as blanks
      line += ' ';
      line += field;
      return;
    }
  }
  // E editing: d.dddddddddddddddde+nnn with a three-digit exponent
  char e[64];
  snprintf(e, sizeof e, "%.16E", v);
  char* p = strchr(e, 'E');
  const int ex = atoi(p + 1);
  *p = '\0';
  snprintf(num, sizeof num, "%sE%c%03d", e, ex < 0 ? '-' : '+', ex < 0 ? -ex : ex);
  snprintf(field, sizeof field, "%25s", num);
  line += ' ';
  line += field;
}

}  // namespace

// OUTPUT (nse_dominik.f:2606-2723) into root/ (root/nseoutput2/... and
// root/temperature_check.dat); cellvalue is (nx,ny,nz,4)
bool write_output_files(const std::string& root, int nx, int ny, int nz, const double* u,
                        const double* v, const double* w, const double* p, const double* x,
                        const double* y, const double* z, const double* T,
                        const double* cellvalue, const double* u_ta, const double* v_ta,
                        const double* w_ta, const double* phi, const double* divu) {
  const std::string od = root + "/nseoutput2";
  if (!ensure_dir(od)) return false;
  const long sx = nx + 2, sy = (long)(nx + 2) * (ny + 2);
  auto P = [&](long i, long j, long k) { return i + sx * j + sy * k; };
  const long nc = (long)nx * ny * nz;
  const char* names[13] = {"velocity", "temperature", "pressure", "divergence", "gridx",
                           "gridy",    "gridz",       "gridnumber", "phi",      "cellvalue1",
                           "cellvalue2", "cellvalue3", "cellvalue4"};
  std::vector<RecWriter*> fw;
  for (const char* n : names) fw.push_back(new RecWriter(od + "/" + n + ".dat"));
  bool ok = true;
  for (auto* f : fw) ok = ok && f->ok;
  if (ok) {
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          double a[3] = {(u[P(i - 1, j, k)] + u[P(i, j, k)]) * 0.50,
                         (v[P(i, j - 1, k)] + v[P(i, j, k)]) * 0.50,
                         (w[P(i, j, k - 1)] + w[P(i, j, k)]) * 0.50};
          for (double& q : a)
            if (fabs(q) < 1.0e-30) q = 0.0;
          const long c = P(i, j, k);
          const long m = (i - 1) + (long)nx * ((j - 1) + (long)ny * (k - 1));
          fw[0]->rec(a, 3);
          fw[2]->rec(p + c, 1);
          fw[1]->rec(T + c, 1);
          fw[3]->rec(divu + c, 1);
          fw[8]->rec(phi + c, 1);
          for (int q = 0; q < 4; ++q) fw[9 + q]->rec(cellvalue + m + q * nc, 1);
        }
    for (int i = 1; i <= nx; ++i) fw[4]->rec(x + i, 1);
    for (int j = 1; j <= ny; ++j) fw[5]->rec(y + j, 1);
    for (int k = 1; k <= nz; ++k) fw[6]->rec(z + k, 1);
    const int32_t n3[3] = {nx, ny, nz};
    fw[7]->rec_ints(n3, 3);
  }
  for (auto* f : fw) {
    ok = f->close() && ok;
    delete f;
  }
  // temperature profile at i = nx, k = nz/2 (list-directed)
  FILE* tc = fopen((root + "/temperature_check.dat").c_str(), "w");
  if (!tc) ok = false;
  else {
    for (int j = 0; j <= ny + 1; ++j) {
      std::string line;
      list_item(line, y[j]);
      list_item(line, T[P(nx, j, nz / 2)]);
      fprintf(tc, "%s\n", line.c_str());
    }
    ok = (fclose(tc) == 0) && ok;
  }
  // field.u (no time record) and grid.u
  {
    RecWriter fu(od + "/field.u");
    ok = ok && fu.ok;
    for (int k = 0; ok && k <= nz + 1; ++k)
      for (int j = 0; j <= ny + 1; ++j)
        for (int i = 0; i <= nx + 1; ++i) {
          const long c = P(i, j, k);
          const double r[9] = {u[c], v[c], w[c], p[c], T[c], phi[c], u_ta[c], v_ta[c], w_ta[c]};
          fu.rec(r, 9);
        }
    ok = fu.close() && ok;
  }
  ok = write_grid_file(od + "/grid.u", nx, ny, nz, x, y, z) && ok;
  if (!ok) set_error(NSE_ERR_ARG, "output: writing the files under %s failed", root.c_str());
  return ok;
}

bool write_grid_file(const std::string& path, int nx, int ny, int nz, const double* x,
                     const double* y, const double* z) {
  RecWriter g(path);
  if (!g.ok) return false;
  for (int i = 1; i <= nx; ++i) g.rec(x + i, 1);
  for (int j = 1; j <= ny; ++j) g.rec(y + j, 1);
  for (int k = 1; k <= nz; ++k) g.rec(z + k, 1);
  return g.close();
}

// field.u of OUTFIELD (with_time: a first record holding tid) or of OUTPUT
bool write_field_file(const std::string& path, bool with_time, double tid, int nx, int ny,
                      int nz, const double* u, const double* v, const double* w,
                      const double* p, const double* T, const double* phi,
                      const double* u_ta, const double* v_ta, const double* w_ta) {
  RecWriter fu(path);
  if (!fu.ok) {
    set_error(NSE_ERR_ARG, "cannot write %s", path.c_str());
    return false;
  }
  if (with_time) fu.rec(&tid, 1);
  const long n = (long)(nx + 2) * (ny + 2) * (nz + 2);
  for (long c = 0; c < n; ++c) {
    const double r[9] = {u[c], v[c], w[c], p[c], T[c], phi[c], u_ta[c], v_ta[c], w_ta[c]};
    fu.rec(r, 9);
  }
  if (!fu.close()) {
    set_error(NSE_ERR_ARG, "writing %s failed", path.c_str());
    return false;
  }
  return true;
}

// READFIELD (nse_dominik.f:2769-2794): field.u without a time record
bool read_field_file(const std::string& path, int nx, int ny, int nz, double* u, double* v,
                     double* w, double* p, double* T, double* phi, double* u_ta, double* v_ta,
                     double* w_ta) {
  RecReader rd(path);
  if (!rd.f) {
    set_error(NSE_ERR_ARG, "cannot open %s", path.c_str());
    return false;
  }
  const long n = (long)(nx + 2) * (ny + 2) * (nz + 2);
  double r[9];
  for (long c = 0; c < n; ++c) {
    if (!rd.rec(r, 9)) {
      set_error(NSE_ERR_ARG, "%s: record %ld is not 9 REAL(8) values", path.c_str(), c + 1);
      return false;
    }
    u[c] = r[0]; v[c] = r[1]; w[c] = r[2]; p[c] = r[3]; T[c] = r[4];
    phi[c] = r[5]; u_ta[c] = r[6]; v_ta[c] = r[7]; w_ta[c] = r[8];
  }
  return true;
}

}  // namespace nse

using namespace nse;

extern "C" {

// OUTPUT, nse_dominik.f:2606 (files under ./nseoutput2 and ./temperature_check.dat)
void output_(const double* u, const double* v, const double* w, const double* p,
             const double* x, const double* y, const double* z, const int* nx, const int* ny,
             const int* nz, const double* T, const double* cellvalue, const double* u_ta,
             const double* v_ta, const double* w_ta, const double* phi, const double* divu) {
  nse_clear_error();
  if (!write_output_files(".", *nx, *ny, *nz, u, v, w, p, x, y, z, T, cellvalue, u_ta, v_ta,
                          w_ta, phi, divu))
    fprintf(stderr, "nsegpu: %s\n", nse_last_error());
}

// OUTFIELD, nse_dominik.f:2726 (./field.u with the time, ./nseoutput2/grid.u)
void outfield_(const double* x, const double* y, const double* z, const double* u,
               const double* v, const double* w, const double* p, const int* nx,
               const int* ny, const int* nz, const double* tid, const double* T,
               const double* phi, const double* u_ta, const double* v_ta,
               const double* w_ta) {
  nse_clear_error();
  bool ok = write_field_file("field.u", true, *tid, *nx, *ny, *nz, u, v, w, p, T, phi, u_ta,
                             v_ta, w_ta);
  ok = ok && ensure_dir_public("nseoutput2") &&
       write_grid_file("nseoutput2/grid.u", *nx, *ny, *nz, x, y, z);
  if (!ok) fprintf(stderr, "nsegpu: %s\n", nse_last_error());
}

// READFIELD, nse_dominik.f:2769 (./nseoutput2/field.u)
void readfield_(double* u, double* v, double* w, double* p, const int* nx, const int* ny,
                const int* nz, double* T, double* phi, double* u_ta, double* v_ta,
                double* w_ta) {
  nse_clear_error();
  if (!read_field_file("nseoutput2/field.u", *nx, *ny, *nz, u, v, w, p, T, phi, u_ta, v_ta,
                       w_ta))
    fprintf(stderr, "nsegpu: %s\n", nse_last_error());
}

}  // extern "C"

namespace nse {
bool ensure_dir_public(const std::string& dir) { return ensure_dir(dir); }
}  // namespace nse
