// clmd_deck.cpp -- the .3d deck reader for hosts without the Fortran
// readdata(): fills the common blocks exactly as read-3d.f:11-302 does
// (fixed columns, version-dependent fields, unit conversion, dmm ring and
// first-passage initialisation).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>

#include "../../include/clmd_f77.h"

namespace {

struct Deck {
  FILE* f = nullptr;
  std::string line;
  bool ok = true;
  bool next() {
    if (!ok) return false;
    char buf[1024];
    if (!fgets(buf, sizeof buf, f)) {
      ok = false;
      line.clear();
      return false;
    }
    line = buf;
    while (!line.empty() && (line.back() == '\n' || line.back() == '\r')) line.pop_back();
    return true;
  }
  // columns [skip, skip+w) with blanks dropped (Fortran BN input)
  std::string field(int skip, int w) const {
    std::string out;
    for (int i = skip; i < skip + w && i < (int)line.size(); i++)
      if (line[i] != ' ' && line[i] != '\t') out += line[i];
    return out;
  }
  // Fw.d: an optional sign, digits with at most one point, an optional
  // exponent (E/D/Q with an optional sign, or a bare sign) and digits;
  // without a point the rightmost d digits are the fraction.  The digits go
  // to strtod as one decimal string (as gfortran converts them), so the
  // value is the correctly rounded one.  Any other field stops the
  // reference's read with a runtime error: here the deck is rejected.
  double F(int skip, int w, int d) {
    next();
    const std::string b = field(skip, w);
    if (b.empty()) return 0.0;
    size_t k = 0;
    std::string sign, dig;
    if (b[k] == '+' || b[k] == '-') sign = b[k++];
    long point = -1;
    for (; k < b.size() && ((b[k] >= '0' && b[k] <= '9') || b[k] == '.'); k++) {
      if (b[k] == '.') {
        if (point >= 0) return bad();
        point = (long)dig.size();
      } else {
        dig += b[k];
      }
    }
    if (dig.empty() || dig.size() > 120) return bad();
    long e = 0;
    if (k < b.size()) {
      if (strchr("eEdDqQ", b[k])) k++;
      else if (b[k] != '+' && b[k] != '-') return bad();
      const bool neg = k < b.size() && b[k] == '-';
      if (k < b.size() && (b[k] == '+' || b[k] == '-')) k++;
      if (k == b.size()) return bad();
      for (; k < b.size(); k++) {
        if (b[k] < '0' || b[k] > '9') return bad();
        if (e < 100000) e = 10 * e + (b[k] - '0');
      }
      if (neg) e = -e;
    }
    if (point < 0) point = (long)dig.size() - d;  // the implied point
    const std::string s = sign + "0." + dig + "e" + std::to_string(e + point);
    return strtod(s.c_str(), nullptr);
  }
  double bad() {
    ok = false;
    return 0.0;
  }
  // Iw: an optional sign and digits (blanks dropped); anything else is a
  // runtime error of the reference's read
  int I(int skip) {
    next();
    const std::string b = field(skip, 10);
    size_t k = (!b.empty() && (b[0] == '+' || b[0] == '-')) ? 1 : 0;
    for (; k < b.size(); k++)
      if (b[k] < '0' || b[k] > '9') {
        ok = false;
        return 0;
      }
    return b.empty() ? 0 : (int)strtol(b.c_str(), nullptr, 10);
  }
  // (41X,A) into CHARACTER*n: n columns from column 42, blank padded
  void A(char* dst, int n) {
    next();
    for (int k = 0; k < n; k++) dst[k] = (41 + k < (int)line.size()) ? line[41 + k] : ' ';
  }
  void skip() { next(); }
};

int fspc(const char* a, int n) {  // read-3d.f:306-319: first blank (1-based), 0 if none
  int p1 = 0;
  for (int i = 1; i <= n; i++)
    if (a[i - 1] == ' ' && p1 == 0) p1 = i;
  return p1;
}

// fx(plen:) = f, Fortran substring assignment (blank padded)
void join(char* fx, int nfx, const char* fpath, int plen, const char* f, int nf) {
  memcpy(fx, fpath, 40 < nfx ? 40 : nfx);
  for (int i = 40; i < nfx; i++) fx[i] = ' ';
  int start = plen > 0 ? plen - 1 : 0;
  for (int i = start, k = 0; i < nfx; i++, k++) fx[i] = k < nf ? f[k] : ' ';
}

}  // namespace

extern "C" int clmd_f77_readdata(const char* path) {
  Deck d;
  d.f = fopen(path, "r");
  if (!d.f) return 1;
  clmd_filep_t& F = filep_;
  clmd_timep_t& T = timep_;
  clmd_boxpp_t& B = boxpp_;
  clmd_atomp_t& P = atomp_;
  clmd_energ_t& E = energ_;
  clmd_dmmpp_t& D = dmmpp_;
  clmd_cvtpp_t& C = cvtpp_;
  const float ver = 1.02f;
  d.skip();
  float fver = (float)d.F(41, 8, 6);
  if (fver < ver) {
    fclose(d.f);
    return 2;
  }
  d.skip();
  d.A(F.fpath, 40);
  int plen = fspc(F.fpath, 40);
  d.A(F.fxyz, 40);
  join(F.fxxyz, 80, F.fpath, plen, F.fxyz, 40);
  F.ftxyz = d.I(41);
  d.A(F.fvel, 40);
  join(F.fxvel, 80, F.fpath, plen, F.fvel, 40);
  F.ftvel = d.I(41);
  d.A(F.facc, 40);
  join(F.fxacc, 80, F.fpath, plen, F.facc, 40);
  F.ftacc = d.I(41);
  d.A(F.frst, 40);
  join(F.fxrst, 80, F.fpath, plen, F.frst, 40);
  F.ftrst = d.I(41);
  d.A(F.fcsi, 40);
  join(F.fxcsi, 80, F.fpath, plen, F.fcsi, 40);
  memset(F.ffpt, ' ', 40);
  memcpy(F.ffpt, "fpt", 3);
  join(F.fxfpt, 80, F.fpath, plen, F.ffpt, 40);
  memset(F.fcsif, ' ', 40);
  memcpy(F.fcsif, "fsi", 3);
  join(F.fxcsif, 80, F.fpath, plen, F.fcsif, 40);
  F.ftcsi = d.I(41);
  d.A(F.fave, 40);
  join(F.fxave, 80, F.fpath, plen, F.fave, 40);
  F.ftave = d.I(41);
  if (fver >= 1.06f) {
    d.A(F.frat, 40);
    join(F.fxrat, 80, F.fpath, plen, F.frat, 40);
    F.ftrat = d.I(41);
  } else {
    F.ftrat = 0;
  }
  C.cstep = -1;
  C.ctrat = F.ftrat;
  C.cen = 0;
  C.ccn = 0;
  d.skip();
  T.dt = d.F(41, 14, 5);
  T.ntim = d.I(40);
  T.btim = d.I(41);
  T.sctim = d.I(41);
  d.skip();
  B.boxx = d.F(41, 14, 5);
  B.boxy = d.F(41, 14, 5);
  B.boxz = d.F(41, 14, 5);
  if (fver >= 1.08f) {
    d.A(&B.bperx, 1);
    d.A(&B.bpery, 1);
    d.A(&B.bperz, 1);
  } else {
    B.bperx = B.bpery = B.bperz = 'X';
  }
  B.bpot = d.F(41, 14, 5);
  B.beng = d.F(41, 14, 5);
  d.A(&B.bcor, 1);
  if (fver >= 1.05f) {
    d.A(&B.bshr, 1);
    B.boxxn = d.F(41, 14, 5);
    B.boxyn = d.F(41, 14, 5);
    B.boxzn = d.F(41, 14, 5);
    B.boxxs = d.F(41, 14, 5);
    B.boxys = d.F(41, 14, 5);
    B.boxzs = d.F(41, 14, 5);
    B.boxt = d.I(41);
  } else {
    B.boxxn = B.boxx;
    B.boxyn = B.boxy;
    B.boxzn = B.boxz;
    B.boxxs = B.boxys = B.boxzs = 0.0;
    B.bshr = '-';
    B.boxt = 1000;
  }
  B.boxx = B.boxx * 10;
  B.boxy = B.boxy * 10;
  B.boxz = B.boxz * 10;
  B.boxxn = B.boxxn * 10;
  B.boxyn = B.boxyn * 10;
  B.boxzn = B.boxzn * 10;
  B.boxxs = fabs(B.boxxs * 10);
  B.boxys = fabs(B.boxys * 10);
  B.boxzs = fabs(B.boxzs * 10);
  B.beng = B.beng * CLMD_CIKB;
  d.skip();
  if (fver < 1.10f) P.atsorts = d.I(41);
  d.A(&F.frctrl, 1);
  d.A(F.finp, 40);
  join(F.fxinp, 80, F.fpath, plen, F.finp, 40);
  d.A(&E.ethst, 1);
  if (fver >= 1.2f) P.Q = d.F(41, 14, 5);
  d.A(&P.rndctrl, 1);
  if (fver >= 1.07f) {
    d.A(&E.eclth, 1);
    E.ecltim = d.I(41);
  } else {
    E.eclth = '-';
    E.ecltim = 1000;
  }
  if (fver >= 1.10f) {
    d.skip();
    P.att = d.F(41, 14, 5);
    P.atskin = d.F(41, 14, 5);
    if (fver >= 1.30f) P.atnenum = d.I(41);
    P.atrcut = d.F(41, 14, 5);
    P.atrskin = d.F(41, 14, 5);
    T.nbtim = d.I(41);
    T.chgNtim = fver >= 1.11f ? d.I(41) : 0;
    if (fver >= 1.12f) {
      d.skip();
      d.A(&C.clnuctrl, 1);
      C.csover = d.I(41);
      C.clwait = d.I(41);
    }
    d.skip();
    P.atsorts = d.I(41);
  }
  d.skip();
  if (fver < 1.10f) {
    d.A(P.apsym[0], 2);
    P.natom = d.I(41);
    P.apmas[0] = d.F(41, 14, 5);
    P.apsig[0] = d.F(41, 14, 5);
    P.apeps[0] = d.F(41, 14, 5);
    P.appr[0] = d.F(41, 14, 5);
    P.appa[0] = d.F(41, 14, 5);
    P.att = d.F(41, 14, 5);
    P.atskin = d.F(41, 14, 5);
    P.atrcut = d.F(41, 14, 5);
    P.atrskin = d.F(41, 14, 5);
    T.nbtim = d.I(41);
    P.apmas[0] = P.apmas[0] * CLMD_CIMU;
    P.apsig[0] = P.apsig[0] * 10.0;
    P.apeps[0] = P.apeps[0] * CLMD_CIKB;
  } else {
    int natom = 1;
    for (int i = 0; i < P.atsorts && i < CLMD_MXSORTS; i++) {
      d.A(P.apsym[i], 2);
      P.apnum[i] = d.I(41);
      P.apmas[i] = d.F(41, 14, 5);
      P.apsig[i] = d.F(41, 14, 5);
      P.apeps[i] = d.F(41, 14, 5);
      P.appr[i] = d.F(41, 14, 5);
      P.appa[i] = d.F(41, 14, 5);
      d.A(&P.apth[i], 1);
      if (fver >= 1.11f) {
        d.A(&P.apNch[i], 1);
        P.apnnum[i] = d.I(41);
      } else {
        P.apNch[i] = '-';
        P.apnnum[i] = P.apnum[i];
      }
      d.skip();
      P.apmas[i] = P.apmas[i] * CLMD_CIMU;
      P.apsig[i] = P.apsig[i] * 10.0;
      P.apeps[i] = P.apeps[i] * CLMD_CIKB;
      for (int j = natom; j <= natom + P.apnum[i] - 1 && j <= CLMD_MXA; j++) {
        P.api[j - 1] = i + 1;
        memcpy(P.apsymi[j - 1], P.apsym[i], 2);
      }
      natom = natom + P.apnum[i];
    }
    P.Q = P.Q * P.apmas[0] * P.apsig[0] * P.apsig[0];
    P.natom = natom - 1;
  }
  // read-3d.f:259-299
  P.atskin = P.atskin * P.apsig[0];
  P.atrcut = P.atrcut * P.apsig[0];
  P.atrskin = P.atrskin * P.apsig[0];
  for (int i = 0; i < 256; i++) D.dmmh[i] = (P.atrskin - P.atrcut) / (double)(float)T.nbtim;
  D.dmmst = 0;
  D.dmmi = 0;
  D.dmmsu = 256.0 * (P.atrskin - P.atrcut) / (double)(float)T.nbtim;
  D.dmms = 0.0;
  E.ewallsum = 0.0;
  E.fwallsum = 0.0;
  C.clookfor = 1;
  C.clookforf = 1;
  C.cbiggest = 0;
  C.cbiggestf = 0;
  int n = P.natom < CLMD_MXA ? P.natom : CLMD_MXA;
  for (int i = 0; i < n; i++) {
    atomc_.x0[i] = atomc_.x1[i] = atomc_.x2[i] = atomc_.x3[i] = atomc_.x4[i] = atomc_.x5[i] = 0.0;
    atomc_.y0[i] = atomc_.y1[i] = atomc_.y2[i] = atomc_.y3[i] = atomc_.y4[i] = atomc_.y5[i] = 0.0;
    atomc_.z0[i] = atomc_.z1[i] = atomc_.z2[i] = atomc_.z3[i] = atomc_.z4[i] = atomc_.z5[i] = 0.0;
    C.cfpt[i] = -1;
    C.cfptf[i] = -1;
  }
  bool ok = d.ok;
  fclose(d.f);
  return ok ? 0 : 3;
}
