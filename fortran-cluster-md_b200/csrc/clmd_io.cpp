// clmd_io.cpp -- restart files and analysis writers in the reference's
// formats, on top of the public C ABI: wrt-rst.f / read-rst.f (gfortran
// unformatted sequential records), wrt-csi.f / wrt-csi-fre.f and wrt-fpt.f
// (Fortran fixed-format text).
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/clmd.h"

namespace {

// ---- gfortran unformatted sequential: [int32 n][n bytes][int32 n] --------
constexpr long long kMaxRecord = 0x7fffffffLL;  // longer records need subrecords
constexpr char kEngineTag[8] = {'C', 'L', 'M', 'D', 'S', 'C', '0', '1'};   // clmd_scalars
constexpr char kReplicaTag[8] = {'C', 'L', 'M', 'D', 'R', 'P', '0', '1'};  // clmd_replica_result

bool put_record(FILE* f, const void* a, size_t na, const void* b = nullptr, size_t nb = 0) {
  const long long n = (long long)(na + nb);
  if (n > kMaxRecord) return false;
  const int32_t m = (int32_t)n;
  if (fwrite(&m, 4, 1, f) != 1) return false;
  if (na && fwrite(a, 1, na, f) != na) return false;
  if (nb && fwrite(b, 1, nb, f) != nb) return false;
  return fwrite(&m, 4, 1, f) == 1;
}

// reads one record into buf; false at end of file or on a malformed frame
bool get_record(FILE* f, std::vector<char>& buf) {
  int32_t m = 0, m2 = 0;
  if (fread(&m, 4, 1, f) != 1 || m < 0) return false;
  buf.resize((size_t)m);
  if (m && fread(buf.data(), 1, (size_t)m, f) != (size_t)m) return false;
  if (fread(&m2, 4, 1, f) != 1 || m2 != m) return false;
  return true;
}

// three arrays of mxa doubles in one record (x0,y0,z0 as wrt-rst.f:39)
bool put_xyz(FILE* f, const double* x, const double* y, const double* z, int n, int mxa,
             std::vector<double>& tmp) {
  tmp.assign((size_t)3 * mxa, 0.0);
  if (x) memcpy(tmp.data(), x, sizeof(double) * n);
  if (y) memcpy(tmp.data() + mxa, y, sizeof(double) * n);
  if (z) memcpy(tmp.data() + 2 * (size_t)mxa, z, sizeof(double) * n);
  return put_record(f, tmp.data(), sizeof(double) * tmp.size());
}

int write_rst_file(const char* path, int n, int mxa, double ekin, double epot,
                   const double* const* xyz /* x0,y0,z0,x1,..,z2 */, const char* tag,
                   const void* eng, size_t eng_bytes) {
  if (!path || n < 1) return CLMD_ERR_ARG;
  if (mxa <= 0) mxa = n;
  if (mxa < n || (long long)mxa * 24 > kMaxRecord) return CLMD_ERR_ARG;
  FILE* f = fopen(path, "wb");
  if (!f) return CLMD_ERR_ARG;
  bool ok = true;
  const int32_t i = mxa;  // wrt-rst.f:35-36 writes mxa, not the step
  const double e5[5] = {ekin, epot, ekin, epot, ekin};
  const double w4[4] = {0.0, 0.0, 0.0, 0.0};  // ewall, ewallsum, fwall, fwallsum
  ok = ok && put_record(f, &i, 4) && put_record(f, e5, sizeof(e5)) && put_record(f, w4, sizeof(w4));
  std::vector<double> tmp;
  for (int k = 0; k < 3 && ok; k++) ok = put_xyz(f, xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2], n, mxa, tmp);
  for (int k = 3; k < 6 && ok; k++) ok = put_xyz(f, nullptr, nullptr, nullptr, n, mxa, tmp);
  if (ok && eng) ok = put_record(f, tag, 8, eng, eng_bytes);
  if (fclose(f) != 0) ok = false;
  return ok ? CLMD_OK : CLMD_ERR_ARG;
}

// ---- Fortran edit descriptors: right-justified, asterisks on overflow ----
void fmt_field(std::string& out, const char* text, int w) {
  const int len = (int)strlen(text);
  if (len > w) {
    out.append((size_t)w, '*');
    return;
  }
  out.append((size_t)(w - len), ' ');
  out.append(text);
}
void fmt_i(std::string& out, long long v, int w) {
  char b[32];
  snprintf(b, sizeof(b), "%lld", v);
  fmt_field(out, b, w);
}
void fmt_f(std::string& out, double v, int w, int d) {
  char b[64];
  if (!isfinite(v)) {
    out.append((size_t)w, '*');
    return;
  }
  snprintf(b, sizeof(b), "%.*f", d, v);
  fmt_field(out, b, w);
}
void sp(std::string& out, int n) { out.append((size_t)n, ' '); }

bool append_text(const char* path, const std::string& s) {
  FILE* f = fopen(path, "ab");
  if (!f) return false;
  bool ok = fwrite(s.data(), 1, s.size(), f) == s.size();
  return fclose(f) == 0 && ok;
}

// wrt-fpt.f:30-37 for one size: Stillinger column in double, tWF column in
// REAL; a tWF size never reached gets the reference's placeholder
// cfptf = INT(REAL(-1) * REAL(dt*1e6)) first
void fpt_line(std::string& out, int i, int cfpt, int cfptf, double dt) {
  const float rdt = (float)(dt * 1.0e6);
  if (cfptf == -1) cfptf = (int)((float)cfptf * rdt);
  fmt_i(out, i, 7);
  sp(out, 3);
  fmt_f(out, (double)(float)cfpt / (dt * 1.0e6), 12, 4);
  sp(out, 3);
  fmt_f(out, (double)((float)cfptf / rdt), 12, 4);
  out += '\n';
}

}  // namespace

extern "C" int clmd_write_rst(clmd_system* sys, const char* path, int32_t mxa) {
  clmd_config cfg;
  int st = clmd_get_config(sys, &cfg);
  if (st) return st;
  const int n = cfg.natom;
  std::vector<double> a((size_t)9 * n);
  double* p[9];
  for (int k = 0; k < 9; k++) p[k] = a.data() + (size_t)k * n;
  clmd_scalars sc;
  st = clmd_get_state(sys, p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8], &sc);
  if (st) return st;
  const double* xyz[9] = {p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8]};
  return write_rst_file(path, n, mxa, sc.ekin, sc.epot, xyz, kEngineTag, &sc, sizeof(sc));
}

extern "C" int clmd_read_rst(clmd_system* sys, const char* path, int32_t* step) {
  clmd_config cfg;
  int st = clmd_get_config(sys, &cfg);
  if (st) return st;
  if (!path) return CLMD_ERR_ARG;
  const int n = cfg.natom;
  FILE* f = fopen(path, "rb");
  if (!f) return CLMD_ERR_ARG;
  std::vector<char> rec;
  int32_t atoms = 0;
  double e5[5] = {0, 0, 0, 0, 0};
  std::vector<double> arr[3];
  bool ok = get_record(f, rec) && rec.size() == 4;
  if (ok) memcpy(&atoms, rec.data(), 4);
  ok = ok && atoms >= n && get_record(f, rec) && rec.size() == sizeof(e5);
  if (ok) memcpy(e5, rec.data(), sizeof(e5));
  ok = ok && get_record(f, rec) && rec.size() == 4 * sizeof(double);  // wall terms
  for (int k = 0; k < 3 && ok; k++) {
    ok = get_record(f, rec) && rec.size() == (size_t)24 * atoms;
    if (ok) {
      arr[k].resize(rec.size() / 8);
      memcpy(arr[k].data(), rec.data(), rec.size());
    }
  }
  for (int k = 3; k < 6 && ok; k++) ok = get_record(f, rec);  // Gear derivatives
  clmd_scalars sc;
  bool have_eng = false;
  if (ok && get_record(f, rec) && rec.size() == sizeof(kEngineTag) + sizeof(sc) &&
      memcmp(rec.data(), kEngineTag, sizeof(kEngineTag)) == 0) {
    memcpy(&sc, rec.data() + sizeof(kEngineTag), sizeof(sc));
    have_eng = true;
  }
  fclose(f);
  if (!ok) return CLMD_ERR_ARG;
  if (!have_eng) {
    st = clmd_get_scalars(sys, &sc);
    if (st) return st;
  }
  sc.ekin = e5[4];  // read-rst.f:43 reads ekin, epot, ekin, epot, ekin
  sc.epot = e5[3];
  const size_t m = (size_t)atoms;
  st = clmd_set_state(sys, arr[0].data(), arr[0].data() + m, arr[0].data() + 2 * m, arr[1].data(),
                      arr[1].data() + m, arr[1].data() + 2 * m, arr[2].data(),
                      arr[2].data() + m, arr[2].data() + 2 * m, nullptr, &sc);
  if (st) return st;
  int32_t s = cfg.btim;  // read-rst.f:61-65
  if (step) *step = s;
  return clmd_neighbor(sys, &s);
}

extern "C" int clmd_write_csi(clmd_system* sys, int32_t step, const char* csi_path,
                              const char* fsi_path) {
  clmd_config cfg;
  int st = clmd_get_config(sys, &cfg);
  if (st) return st;
  if (!csi_path) return CLMD_ERR_ARG;
  const int n = cfg.natom;
  std::vector<int32_t> csi(n + 1), csif(n + 1), cgsa(n), cgsfa(n + 1);
  std::vector<double> ceks(n + 1), ceksf(n + 1);
  clmd_cluster_view v;
  memset(&v, 0, sizeof(v));
  v.csi = csi.data();
  v.ceks = ceks.data();
  v.csif = csif.data();
  v.ceksf = ceksf.data();
  v.cgsa = cgsa.data();
  v.cgsfa = cgsfa.data();
  st = clmd_get_clusters(sys, &v);
  if (st) return st;
  const double cikb = CLMD_CIKB;
  const bool fre = cfg.clustering == CLMD_CLU_FRENKEL;
  std::string a, b;
  fmt_i(a, step, 15);
  a += '\n';
  if (fre && fsi_path) {
    // wrt-csi-fre.f:33-43: the monomer line of the tWF file
    fmt_i(b, step, 15);
    b += '\n';
    sp(b, 3);
    fmt_i(b, 0, 7);
    sp(b, 3);
    fmt_i(b, csif[0], 7);
    sp(b, 3);
    fmt_f(b, 0.0, 7, 3);
    sp(b, 3);
    if (csif[0] == 0) {
      fmt_f(b, 0.0, 17, 15);
      sp(b, 3);
      fmt_f(b, 0.0, 10, 5);
    } else {
      fmt_f(b, ceksf[0] / (double)csif[0], 17, 15);
      sp(b, 3);
      fmt_f(b, ceksf[0] / ((double)csif[0] * 1.5 * cikb), 10, 5);
    }
    b += '\n';
  }
  for (int i = 1; i <= n; i++) {
    if (csi[i] != 0) {
      // wrt-csi.f:30-35; wrt-csi-fre.f:46-50 adds REAL(cgsa(i))/REAL(csi(i))
      const double den = (double)((long long)i * csi[i]);
      sp(a, 3);
      fmt_i(a, i, 7);
      sp(a, 3);
      fmt_i(a, csi[i], 7);
      if (fre) {
        sp(a, 3);
        fmt_f(a, (double)((float)cgsa[i - 1] / (float)csi[i]), 7, 3);
      }
      sp(a, 3);
      fmt_f(a, ceks[i] / den, 17, 15);
      sp(a, 3);
      fmt_f(a, ceks[i] / (den * 1.5 * cikb), 10, 5);
      a += '\n';
    }
    if (fre && fsi_path && csif[i] != 0) {
      // wrt-csi-fre.f:52-56: all in REAL
      const long long ic = (long long)i * csif[i];
      sp(b, 3);
      fmt_i(b, i, 7);
      sp(b, 3);
      fmt_i(b, csif[i], 7);
      sp(b, 3);
      fmt_f(b, (double)((float)cgsfa[i] / (float)csif[i]), 7, 3);
      sp(b, 3);
      fmt_f(b, (double)((float)ceksf[i] / (float)ic), 17, 15);
      sp(b, 3);
      fmt_f(b, (double)((float)ceksf[i] / (float)((double)ic * 1.5 * cikb)), 10, 5);
      b += '\n';
    }
  }
  if (!append_text(csi_path, a)) return CLMD_ERR_ARG;
  if (fre && fsi_path && !append_text(fsi_path, b)) return CLMD_ERR_ARG;
  return CLMD_OK;
}

extern "C" int clmd_write_fpt(clmd_system* sys, const char* path) {
  clmd_config cfg;
  int st = clmd_get_config(sys, &cfg);
  if (st) return st;
  if (!path) return CLMD_ERR_ARG;
  const int n = cfg.natom;
  std::vector<int32_t> cfpt(n), cfptf(n);
  clmd_cluster_view v;
  memset(&v, 0, sizeof(v));
  v.cfpt = cfpt.data();
  v.cfptf = cfptf.data();
  st = clmd_get_clusters(sys, &v);
  if (st) return st;
  std::string out;
  for (int i = 1; i <= n; i++)
    if (cfpt[i - 1] != -1) fpt_line(out, i, cfpt[i - 1], cfptf[i - 1], cfg.dt);
  return append_text(path, out) ? CLMD_OK : CLMD_ERR_ARG;
}

extern "C" int clmd_ens_write_rst(clmd_ensemble* e, int32_t slot, const char* path,
                                  int32_t mxa) {
  if (!e || !path) return CLMD_ERR_ARG;
  clmd_replica_result r;
  bool found = false;
  std::vector<clmd_replica_result> res(1024);
  int32_t nres = 0;
  int st = clmd_ens_results(e, res.data(), (int32_t)res.size(), &nres);
  if (st) return st;
  if (nres > (int32_t)res.size()) {
    res.resize(nres);
    st = clmd_ens_results(e, res.data(), nres, &nres);
    if (st) return st;
  }
  for (int k = 0; k < nres; k++)
    if (res[k].slot == slot) {
      r = res[k];
      found = true;
    }
  if (!found) return CLMD_ERR_ARG;
  const int n = r.natom;
  std::vector<double> a((size_t)9 * n);
  double* p[9];
  for (int k = 0; k < 9; k++) p[k] = a.data() + (size_t)k * n;
  st = clmd_ens_get_state(e, slot, p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8],
                          nullptr);
  if (st) return st;
  const double* xyz[9] = {p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8]};
  return write_rst_file(path, n, mxa, r.ekin, r.epot, xyz, kReplicaTag, &r, sizeof(r));
}

extern "C" int clmd_ens_write_fpt(clmd_ensemble* e, int32_t slot, double dt, const char* path) {
  if (!e || !path) return CLMD_ERR_ARG;
  std::vector<int32_t> fpt(4096);
  int st = clmd_ens_fpt(e, slot, fpt.data(), (int32_t)fpt.size());
  if (st) return st;
  std::string out;
  for (int i = 1; i <= (int)fpt.size(); i++)
    if (fpt[i - 1] != -1) fpt_line(out, i, fpt[i - 1], -1, dt);
  return append_text(path, out) ? CLMD_OK : CLMD_ERR_ARG;
}
