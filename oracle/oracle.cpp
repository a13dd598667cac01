// FP64 CPU restatement of the reference's GCM timestep (the parity oracle).
//
// TEST INFRASTRUCTURE. Only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg load this library; the product path never links it.
//
// Each function below restates one WGSL compute kernel of
// ryoung48/web-exoplasim (paths relative to src/model/climate/gcm/) as a plain
// loop over that kernel's threads, evaluated in double precision, in the
// dispatch order of stepper/index.ts:148-161 and dynamics/index.ts:171-344.
// State and tables live in named arrays of `real` with the reference's layouts
// (spectral [plane][NRSP], Fourier [plane][lat][NFC], grid [plane][NHOR]).
// The reference's WGSL helpers precise_log/exp/pow/divide/atan are f32
// accuracy fixes; in f64 they are the plain libm functions.
//
// Sequential-f32 mode. Built with -DORACLE_REAL=float and
// -fsingle-precision-constant (liboracle32.so), the same loops run with every
// value, constant, table and intermediate in f32 and the f32 libm routines.
// That is the comparator of the reference's gates
// (scripts/exoplasim-webgpu/verify-kernels.mjs:273, "<= 2x sequential f32",
// and verify-dynamics.mjs:179-181, V3: the GPU's error against f64 within
// twice that of an f32 build replaying the same routine from the same state).
// The C interface below exchanges doubles in both builds; the f32 build rounds
// what it is given once, as the GPU's f32 state and tables are rounded.
#ifndef ORACLE_REAL
#define ORACLE_REAL double
#endif
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "oracle_fields.h"

namespace {

using real = ORACLE_REAL;

// Every kernel constant, under the reference's WGSL override names.
#define ORACLE_CONSTS(X)                                                                          \
  X(PSURF) X(WW) X(CV) X(CT) X(AKAP) X(RDBRV) X(ADV) X(ACPD) X(GA) X(GASCON) X(PLAVOR) X(DELT)    \
  X(DELT2) X(DELTSEC) X(DELTSEC2) X(PNU) X(PNU21) X(FILTER) X(RA1) X(RA2) X(RA4) X(TMELT) X(ALV)  \
  X(ALS) X(MOIST) X(ZUMIN) X(VDIFF_B) X(VDIFF_C) X(VDIFF_D) X(NDHEAT) X(NFIXED) X(ZRLON) X(ZDAWN) \
  X(OZONE) X(A0O3) X(A1O3) X(ACO3) X(BO3) X(CO3) X(ZCONST) X(GSOL0) X(ZSOLAR1) X(ZSOLAR2)         \
  X(ZSOLARS1) X(ZSOLARS2) X(TSWR1) X(TSWR2) X(TSWR3) X(ZB3) X(ZB4) X(ZB5) X(RCOEFF)               \
  X(LN_DIFFUSE_RAYLEIGH) X(NSTARTEMP) X(SBK) X(TH2OC) X(TPOFMT) X(ZFCO2_ZZF2) X(ZAO30) X(ZCO20)   \
  X(ZH2O0A) X(ZH2O0) X(ZAO3C) X(ZACO2C) X(ZAH2OC) X(ZTH2OC) X(RHBETA) X(NBETA) X(PDEEP)           \
  X(PDEEPTH) X(RKSHALLOW) X(GAMMA) X(ZRFAC) X(CLWFAC) X(CLWCRIT1) X(CLWCRIT2) X(SICECAP)          \
  X(SOILCAP) X(SICEDIFF) X(SOILDIFF) X(SNOWCAP) X(SNOWDIFF) X(RHOSNOW) X(DZTOP) X(DSMAX)          \
  X(ALBSMAX) X(ALBSMIN) X(ALBSMAXF) X(ALBSMINF) X(ALBSMAX1) X(ALBSMIN1) X(ALBSMAXF1) X(ALBSMINF1) \
  X(ALBSMAX2) X(ALBSMIN2) X(ALBSMAXF2) X(ALBSMINF2) X(ALBGMAX) X(ALBGMIN) X(ALBGMAX1) X(ALBGMIN1) \
  X(ALBGMAX2) X(ALBGMIN2) X(DRHSFULL) X(NWETSOIL) X(WSMAX) X(ALBLAND) X(ALBLANDMAX)               \
  X(DGROUNDALB1) X(DGROUNDALB2) X(DOCEANALB1) X(DOCEANALB2) X(NVEG) X(RLUE) X(CO2CONV) X(TAU_VEG) \
  X(TAU_SOIL) X(VWS_CRIT) X(Q10) X(ZLAIMAX) X(ZLAIMIN) X(VALB_MIN) X(VALB_MAX) X(VSALB_MIN)       \
  X(VWMAX_MAX) X(VWMAX_MIN) X(VZ0_MIN) X(CVEG_A) X(CVEG_C) X(CVEG_F) X(CVEG_K) X(CVEG_L)          \
  X(CT_CRIT) X(CO2_REF) X(CO2_COMP) X(CO2_SENS) X(CVEG_E) X(CVEG_G) X(NCVEG) X(NGLACIER)         \
  X(GLACELIM) X(XDT) X(XMIND) X(XMAXD) X(CICEMIN) X(THICEC) X(TFREEZE) X(CRHOI) X(CRHOS)         \
  X(CRHOSN) X(CPI) X(CKAPI) X(CKAPSN) X(CLFI) X(CLFSN) X(DTMIX) X(CPS) X(CHARNOCK) X(DZ0SEA)     \
  X(DZ0ICE) X(DRHSSEA) X(DRHSICE) X(ALBSEA) X(ALBICE) X(DICEALBMX1) X(DICEALBMX2) X(DICEALBMN1)  \
  X(DICEALBMN2) X(ICE_COUPLED) X(NCARBON) X(NSUPPLY) X(TIMEWEIGHT) X(CO2EARTH) X(BETA) X(KACT)   \
  X(PEARTH) X(WMAX) X(VEARTH) X(PLARAD) X(RAD_EARTHSQ) X(JET) X(SIGMA_LOW) X(NSTORMDIAG) X(CKCD)   \
  X(VITHRESH)

struct Consts {
#define DECL(n) real n = 0;
  ORACLE_CONSTS(DECL)
#undef DECL
};

constexpr int MAXL = 32;
using Vec = std::vector<real>;

struct Model {
  int T, L, NLAT, NLON, NHOR, NTP1, NCSP, NRSP, NFC, NLEV, NLEM, NLEP;
  Consts k;
  std::map<std::string, Vec> state;
  std::map<std::string, Vec> tables;

  Model(int t, int l) : T(t), L(l) {
    NLAT = t == 21 ? 32 : t == 42 ? 64 : t == 63 ? 96 : 0;
    if (!NLAT || l < 2 || l > MAXL) throw std::runtime_error("unsupported resolution");
    NLON = 2 * NLAT;
    NHOR = NLAT * NLON;
    NTP1 = t + 1;
    NCSP = NTP1 * (NTP1 + 1) / 2;
    NRSP = 2 * NCSP;
    NFC = 2 * NTP1;
    NLEV = l;
    NLEM = l - 1;
    NLEP = l + 1;
    const int P = 51 + 5 * l;
    const int S_ = NRSP, F_ = NLAT * NFC, G_ = NHOR, T_ = 1, H = l + 1, L_ = l;
    (void)P; (void)S_; (void)F_; (void)G_; (void)T_; (void)H; (void)L_;
#define MAKE(name, shape, count) state[#name] = Vec((size_t)shape##_ * (count), 0.0);
    {
      const int L = L_;
      (void)L;
      ORACLE_FIELDS(MAKE)
    }
#undef MAKE
  }
  real* F(const char* n) {
    auto it = state.find(n);
    if (it == state.end()) throw std::runtime_error(std::string("no field ") + n);
    return it->second.data();
  }
  const real* TB(const char* n) {
    auto it = tables.find(n);
    if (it == tables.end()) throw std::runtime_error(std::string("no table ") + n);
    return it->second.data();
  }
  int planes(const char* n) {
    auto& v = state.at(n);
    return (int)v.size();
  }
};

// ----------------------------------------------------------------- transforms
// fourier/wgsl/forward.wgsl:1-18 (gp2fc): c[k] = sum_j table[j][k] g[j].
void fourier_forward(Model& m, const char* src, const char* dst, int planes) {
  const real* tab = m.TB("fourier_forward");
  const real* g = m.F(src);
  real* c = m.F(dst);
  for (int row = 0; row < planes * m.NLAT; ++row)
    for (int k = 0; k < m.NFC; ++k) {
      real s = 0;
      for (int j = 0; j < m.NLON; ++j) s += tab[j * m.NFC + k] * g[row * m.NLON + j];
      c[row * m.NFC + k] = s;
    }
}

// fourier/wgsl/inverse.wgsl:1-18 (fc2gp): g[j] = sum_k table[k][j] c[k].
void fourier_inverse(Model& m, const char* src, const char* dst, int planes) {
  const real* tab = m.TB("fourier_inverse");
  const real* c = m.F(src);
  real* g = m.F(dst);
  for (int row = 0; row < planes * m.NLAT; ++row)
    for (int j = 0; j < m.NLON; ++j) {
      real s = 0;
      for (int k = 0; k < m.NFC; ++k) s += tab[k * m.NLON + j] * c[row * m.NFC + k];
      g[row * m.NLON + j] = s;
    }
}

// fourier/wgsl/dlambda.wgsl:1-17: (re, im) * i m.
void fourier_dlambda(Model& m, const char* src, const char* dst, int planes) {
  const real* a = m.F(src);
  real* b = m.F(dst);
  for (int i = 0; i < planes * m.NLAT * m.NTP1; ++i) {
    int mm = i % m.NTP1;
    int at = (i / m.NTP1) * m.NFC + 2 * mm;
    real re = a[at], im = a[at + 1];
    b[at] = -im * mm;
    b[at + 1] = re * mm;
  }
}

static void mode_of(const Model& m, int w, int& mm, int& n) {
  int start = 0;
  mm = 0;
  while (w >= start + m.NTP1 - mm) {
    start += m.NTP1 - mm;
    mm++;
  }
  n = mm + w - start;
}

// legendre/wgsl/forward.wgsl:1-38 (fc2sp, single-process branch).
void legendre_forward(Model& m, const char* src, const char* dst, const char* table, int planes) {
  const real* q = m.TB(table);
  const real* f = m.F(src);
  real* s = m.F(dst);
  for (int p = 0; p < planes; ++p)
    for (int w = 0; w < m.NCSP; ++w) {
      int mm, n;
      mode_of(m, w, mm, n);
      real sign = (mm + n) % 2 == 0 ? 1.0 : -1.0;
      const real* four = f + (size_t)p * m.NLAT * m.NFC + 2 * mm;
      real re = 0, im = 0;
      for (int l = 0; l < m.NLAT / 2; ++l) {
        real qq = q[l * m.NCSP + w];
        const real* north = four + l * m.NFC;
        const real* south = four + (m.NLAT - 1 - l) * m.NFC;
        re += qq * (north[0] + sign * south[0]);
        im += qq * (north[1] + sign * south[1]);
      }
      s[(size_t)p * m.NRSP + 2 * w] = re;
      s[(size_t)p * m.NRSP + 2 * w + 1] = im;
    }
}

// legendre/wgsl/inverse.wgsl:1-27 (sp2fc, sp2fcdmu).
void legendre_inverse(Model& m, const char* src, const char* dst, const char* table, int planes) {
  const real* q = m.TB(table);
  const real* s = m.F(src);
  real* f = m.F(dst);
  for (int i = 0; i < planes * m.NLAT * m.NTP1; ++i) {
    int mm = i % m.NTP1;
    int row = i / m.NTP1;
    int plane = row / m.NLAT, lat = row % m.NLAT;
    int first = mm * (2 * m.NTP1 - mm + 1) / 2;
    const real* sp = s + (size_t)plane * m.NRSP;
    real re = 0, im = 0;
    for (int w = first; w < first + m.NTP1 - mm; ++w) {
      real qq = q[lat * m.NCSP + w];
      re += qq * sp[2 * w];
      im += qq * sp[2 * w + 1];
    }
    f[(size_t)row * m.NFC + 2 * mm] = re;
    f[(size_t)row * m.NFC + 2 * mm + 1] = im;
  }
}

// legendre/wgsl/dv2uv.wgsl:1-43.
void legendre_dv2uv(Model& m, const char* dname, const char* zname, const char* uname,
                    const char* vname, int planes, real plavor) {
  const real* qu = m.TB("legendre_qu");
  const real* qv = m.TB("legendre_qv");
  const real* D = m.F(dname);
  const real* Z = m.F(zname);
  real* U = m.F(uname);
  real* V = m.F(vname);
  for (int i = 0; i < planes * m.NLAT * m.NTP1; ++i) {
    int mm = i % m.NTP1;
    int row = i / m.NTP1;
    int plane = row / m.NLAT, lat = row % m.NLAT;
    int first = mm * (2 * m.NTP1 - mm + 1) / 2;
    const real* d = D + (size_t)plane * m.NRSP;
    const real* z = Z + (size_t)plane * m.NRSP;
    real ure = 0, uim = 0, vre = 0, vim = 0;
    for (int w = first; w < first + m.NTP1 - mm; ++w) {
      real a = qu[lat * m.NCSP + w], b = qv[lat * m.NCSP + w];
      real zre = w == 1 ? z[2 * w] - plavor : z[2 * w];
      real zim = z[2 * w + 1], dre = d[2 * w], dim = d[2 * w + 1];
      ure = ure + b * zre + a * dim;
      uim = uim + b * zim - a * dre;
      vre = vre + a * zim - b * dre;
      vim = vim - a * zre - b * dim;
    }
    size_t at = (size_t)row * m.NFC + 2 * mm;
    U[at] = ure;
    U[at + 1] = uim;
    V[at] = vre;
    V[at + 1] = vim;
  }
}

// legendre/wgsl/uv2dv.wgsl:1-63 (uv2dv; mktend's with the kinetic term).
void legendre_uv2dv(Model& m, const char* uname, const char* vname, const char* kname,
                    const char* dname, const char* zname, int planes) {
  const real* qe = m.TB("legendre_qe");
  const real* qm = m.TB("legendre_qm");
  const real* qqt = m.TB("legendre_qq");
  const real* U = m.F(uname);
  const real* V = m.F(vname);
  const real* K = kname ? m.F(kname) : nullptr;
  real* D = m.F(dname);
  real* Z = m.F(zname);
  for (int p = 0; p < planes; ++p)
    for (int w = 0; w < m.NCSP; ++w) {
      int mm, n;
      mode_of(m, w, mm, n);
      real s = (mm + n) % 2 == 0 ? 1.0 : -1.0;
      size_t column = (size_t)p * m.NLAT * m.NFC + 2 * mm;
      real dre = 0, dim = 0, zre = 0, zim = 0;
      for (int l = 0; l < m.NLAT / 2; ++l) {
        size_t north = column + l * m.NFC, south = column + (m.NLAT - 1 - l) * m.NFC;
        real e = qe[l * m.NCSP + w], mq = qm[l * m.NCSP + w];
        real dure = U[north] - s * U[south], duim = U[north + 1] - s * U[south + 1];
        real dvre = V[north] - s * V[south], dvim = V[north + 1] - s * V[south + 1];
        real sure = U[north] + s * U[south], suim = U[north + 1] + s * U[south + 1];
        real svre = V[north] + s * V[south], svim = V[north + 1] + s * V[south + 1];
        if (K) {
          real q2 = qqt[l * m.NCSP + w];
          dre = dre + q2 * (K[north] + s * K[south]);
          dim = dim + q2 * (K[north + 1] + s * K[south + 1]);
        }
        dre = dre - e * dvre - mq * suim;
        dim = dim - e * dvim + mq * sure;
        zre = zre + e * dure - mq * svim;
        zim = zim + e * duim + mq * svre;
      }
      size_t at = (size_t)p * m.NRSP + 2 * w;
      D[at] = dre;
      D[at + 1] = dim;
      Z[at] = zre;
      Z[at + 1] = zim;
    }
}

// legendre/wgsl/qtend.wgsl:1-46.
void legendre_qtend(Model& m, const char* uname, const char* vname, const char* srcname,
                    const char* dst, int planes) {
  const real* qe = m.TB("legendre_qe");
  const real* qc = m.TB("legendre_qc");
  const real* qm = m.TB("legendre_qm");
  const real* U = m.F(uname);
  const real* V = m.F(vname);
  const real* Sx = m.F(srcname);
  real* out = m.F(dst);
  for (int p = 0; p < planes; ++p)
    for (int w = 0; w < m.NCSP; ++w) {
      int mm, n;
      mode_of(m, w, mm, n);
      real s = (mm + n) % 2 == 0 ? 1.0 : -1.0;
      size_t column = (size_t)p * m.NLAT * m.NFC + 2 * mm;
      real re = 0, im = 0;
      for (int l = 0; l < m.NLAT / 2; ++l) {
        size_t north = column + l * m.NFC, south = column + (m.NLAT - 1 - l) * m.NFC;
        real e = qe[l * m.NCSP + w], c = qc[l * m.NCSP + w], mq = qm[l * m.NCSP + w];
        re = re + e * (V[north] - s * V[south]) + c * (Sx[north] + s * Sx[south]) +
             mq * (U[north + 1] + s * U[south + 1]);
        im = im + e * (V[north + 1] - s * V[south + 1]) + c * (Sx[north + 1] + s * Sx[south + 1]) -
             mq * (U[north] + s * U[south]);
      }
      out[(size_t)p * m.NRSP + 2 * w] = re;
      out[(size_t)p * m.NRSP + 2 * w + 1] = im;
    }
}

// ----------------------------------------------------------------- dynamics
// dynamics/wgsl/calcgp.wgsl:1-147.
void calcgp(Model& m) {
  const Consts& K = m.k;
  const int NL = m.NLEV, NH = m.NHOR;
  const real *rcsqT = m.TB("rcsq"), *t0T = m.TB("t0"), *ds = m.TB("dsigma"), *sh = m.TB("sigmah");
  const real *rd = m.TB("rdsig"), *t01 = m.TB("t01s2"), *tkpT = m.TB("tkp"), *C = m.TB("c"),
               *G = m.TB("g");
  real *GP = m.F("gp"), *GPMT = m.F("gpmt"), *GPJ = m.F("gpj"), *GU = m.F("gu"), *GV = m.F("gv"),
         *GT = m.F("gt"), *GD = m.F("gd"), *GZ = m.F("gz"), *GQ = m.F("gq");
  real *GTN = m.F("gtn"), *GQN = m.F("gqn"), *GUZ = m.F("guz"), *GVZ = m.F("gvz"), *DW = m.F("dw"),
         *GUT = m.F("gut"), *GVT = m.F("gvt"), *GKE = m.F("gke"), *GUQ = m.F("guq"), *GVQ = m.F("gvq"),
         *DU0 = m.F("du0"), *DV0 = m.F("dv0"), *GVPP = m.F("gvpp"), *DP0 = m.F("dp0");
  for (int h = 0; h < NH; ++h) {
    real rcsq = rcsqT[h];
    real ps = std::exp(GP[h]);
    GP[h] = ps;
    real gpm = GPMT[h], gpj = GPJ[h];
    real gu[MAXL], gv[MAXL], gt[MAXL], gd[MAXL], gz[MAXL], gq[MAXL], zvgpg[MAXL], ztv1[MAXL],
        ztv2[MAXL];
    for (int l = 0; l < NL; ++l) {
      int at = l * NH + h;
      gu[l] = GU[at];
      gv[l] = GV[at];
      gt[l] = GT[at];
      gd[l] = GD[at];
      gz[l] = GZ[at];
      gq[l] = GQ[at];
      zvgpg[l] = rcsq * (gu[l] * gpm + gv[l] * gpj);
      real zq = std::max(gq[l] / ps, 0.0);
      real t0 = t0T[l];
      real tvirt = (gt[l] + t0) * (1.0 + (1.0 / K.RDBRV - 1.0) * zq);
      ztv1[l] = tvirt - t0;
      ztv2[l] = tvirt / (1.0 + K.ADV * zq) - t0;
    }
    real zsdotp[MAXL];
    real zsumd = ds[0] * gd[0];
    real gvp = ds[0] * zvgpg[0];
    zsdotp[0] = zsumd + gvp;
    for (int l = 1; l < NL - 1; ++l) {
      zsumd = zsumd + ds[l] * gd[l];
      gvp = gvp + ds[l] * zvgpg[l];
      zsdotp[l] = zsumd + gvp;
    }
    zsumd = zsumd + ds[NL - 1] * gd[NL - 1];
    gvp = gvp + ds[NL - 1] * zvgpg[NL - 1];
    real gtd[MAXL], gqm[MAXL], gud[MAXL], gvd[MAXL];
    for (int l = 0; l < NL - 1; ++l) {
      zsdotp[l] = sh[l] * (zsumd + gvp) - zsdotp[l];
      gtd[l] = zsdotp[l] * (gt[l + 1] - gt[l]);
      gqm[l] = zsdotp[l] * (gq[l + 1] + gq[l]);
      gud[l] = zsdotp[l] * (gu[l + 1] - gu[l]);
      gvd[l] = zsdotp[l] * (gv[l + 1] - gv[l]);
    }
    real gtn[MAXL], gqn[MAXL], guz[MAXL], gvz[MAXL], dw[MAXL];
    zsumd = zvgpg[0] * ds[0];
    real rdsig0 = rd[0];
    gtn[0] = gt[0] * gd[0] - K.AKAP * ztv2[0] * gd[0] -
             rdsig0 * (gtd[0] + t01[0] * (sh[0] * gvp - zsumd));
    gqn[0] = -rdsig0 * gqm[0];
    guz[0] = -gu[0] * gz[0] - gpj * ztv1[0] - rdsig0 * gvd[0];
    gvz[0] = gv[0] * gz[0] - gpm * ztv1[0] - rdsig0 * gud[0];
    dw[0] = gd[0] * ps * K.PSURF * K.WW;
    for (int l = 1; l < NL; ++l) {
      int column = l * NL;
      real ztpta = C[column] * zvgpg[0];
      real ztptb = C[column] * (zvgpg[0] + gd[0]);
      for (int j = 1; j <= l; ++j) {
        ztpta = ztpta + C[column + j] * zvgpg[j];
        ztptb = ztptb + C[column + j] * (zvgpg[j] + gd[j]);
      }
      real rdsig = rd[l], t01s2 = t01[l], t01s2m = t01[l - 1], sigmah = sh[l], sigmahm = sh[l - 1];
      real tkp = tkpT[l];
      if (l < NL - 1) {
        zsumd = zsumd + zvgpg[l] * ds[l];
        gtn[l] = gt[l] * gd[l] + K.AKAP * ztv2[l] * (zvgpg[l] - ztptb) + tkp * (zvgpg[l] - ztpta) -
                 rdsig * (gtd[l] + gtd[l - 1] + gvp * (t01s2 * sigmah + t01s2m * sigmahm) -
                          zsumd * (t01s2m + t01s2) + zvgpg[l] * ds[l] * t01s2m);
        gqn[l] = -rdsig * (gqm[l] - gqm[l - 1]);
        guz[l] = -gu[l] * gz[l] - gpj * ztv1[l] - rdsig * (gvd[l] + gvd[l - 1]);
        gvz[l] = gv[l] * gz[l] - gpm * ztv1[l] - rdsig * (gud[l] + gud[l - 1]);
      } else {
        gtn[l] = gt[l] * gd[l] + K.AKAP * ztv2[l] * (zvgpg[l] - ztptb) + tkp * (zvgpg[l] - ztpta) -
                 rdsig * (gtd[NL - 2] + t01s2m * (sigmahm * gvp - zsumd));
        gqn[l] = rdsig * gqm[NL - 2];
        guz[l] = -gu[l] * gz[l] - gpj * ztv1[l] - rdsig * gvd[NL - 2];
        gvz[l] = gv[l] * gz[l] - gpm * ztv1[l] - rdsig * gud[NL - 2];
      }
      dw[l] = (zvgpg[l] - ztptb) * ps * K.PSURF * K.WW;
    }
    real scale = std::sqrt(rcsq);
    for (int l = 0; l < NL; ++l) {
      real gsum = 0;
      for (int kk = 0; kk < NL; ++kk) gsum = gsum + G[l * NL + kk] * (ztv1[kk] - gt[kk]);
      real gphi = gsum * 2.0 / rcsq;
      int at = l * NH + h;
      GTN[at] = gtn[l];
      GQN[at] = gqn[l];
      GUZ[at] = guz[l];
      GVZ[at] = gvz[l];
      DW[at] = dw[l];
      GUT[at] = gu[l] * gt[l];
      GVT[at] = gv[l] * gt[l];
      GKE[at] = gu[l] * gu[l] + gv[l] * gv[l] + gphi;
      GUQ[at] = gu[l] * gq[l];
      GVQ[at] = gv[l] * gq[l];
      DU0[at] = K.CV * gu[l] * scale;
      DV0[at] = K.CV * gv[l] * scale;
    }
    GVPP[h] = gvp;
    DP0[h] = K.PSURF * ps;
  }
}

// dynamics/wgsl/spectrala.wgsl:1-109.
void spectrala(Model& m) {
  const Consts& K = m.k;
  const int NL = m.NLEV, NR = m.NRSP;
  const real *G = m.TB("g"), *t0T = m.TB("t0"), *sop = m.TB("sop"), *nidx = m.TB("nindex"),
               *bm1 = m.TB("bm1"), *ds = m.TB("dsigma"), *tau = m.TB("tau");
  real *SPM = m.F("spm"), *SPT = m.F("spt"), *SPP = m.F("spp"), *SP = m.F("sp");
  real *SDM = m.F("sdm"), *SZM = m.F("szm"), *STM = m.F("stm"), *SQM = m.F("sqm"), *SDT = m.F("sdt"),
         *STT = m.F("stt"), *SZT = m.F("szt"), *SQT = m.F("sqt"), *SDP = m.F("sdp"), *STP = m.F("stp"),
         *SZP = m.F("szp"), *SQP = m.F("sqp"), *SD = m.F("sd"), *ST = m.F("st"), *SZ = m.F("sz"),
         *SQ = m.F("sq");
  bool filter = K.FILTER != 0;
  for (int s = 0; s < NR; ++s) {
    real apm = SPM[s];
    real adm[MAXL], azm[MAXL], atm[MAXL], aqm[MAXL], adt[MAXL], stt[MAXL];
    for (int l = 0; l < NL; ++l) {
      int at = l * NR + s;
      adm[l] = SDM[at];
      azm[l] = SZM[at];
      atm[l] = STM[at];
      aqm[l] = SQM[at];
      adt[l] = SDT[at];
      stt[l] = STT[at];
    }
    real zgt[MAXL], zgm[MAXL];
    for (int l = 0; l < NL; ++l) {
      real gt = 0, gm = 0;
      for (int kk = 0; kk < NL; ++kk) {
        gt = gt + G[l * NL + kk] * stt[kk];
        gm = gm + G[l * NL + kk] * atm[kk];
      }
      zgt[l] = gt;
      zgm[l] = gm;
    }
    real spt = SPT[s];
    real spm = apm;
    real so = sop[s];
    int jn = (int)nidx[s];
    real sdt[MAXL];
    for (int l = 0; l < NL; ++l) {
      real zsum = 0;
      if (jn > 0) {
        real zq = 1.0 / (real)(jn * (jn + 1));
        for (int l2 = 0; l2 < NL; ++l2) {
          real z0 = t0T[l2];
          real zt = zgt[l2] - z0 * spt;
          real zm = zgm[l2] + z0 * spm;
          real za = adt[l2] * zq + so;
          real zb = adm[l2] * zq;
          real zz = zb + K.DELT * (zm + za + K.DELT * zt);
          zsum = zsum + zz * bm1[((jn - 1) * NL + l) * NL + l2];
        }
      }
      sdt[l] = s < 2 ? 0.0 : zsum;
    }
    for (int l = 0; l < NL; ++l) spt = spt + ds[l] * sdt[l];
    for (int l = 0; l < NL; ++l) {
      real t = 0;
      for (int kk = 0; kk < NL; ++kk) t = t + tau[l * NL + kk] * sdt[kk];
      stt[l] = stt[l] - t;
    }
    real spp = SPP[s];
    if (filter) SPM[s] = K.PNU21 * spp + K.PNU * apm;
    real sppNew = s < 2 ? 0.0 : apm - K.DELT2 * spt;
    SPP[s] = sppNew;
    SP[s] = sppNew;
    SPT[s] = spt;
    for (int l = 0; l < NL; ++l) {
      int at = l * NR + s;
      if (filter) {
        SDM[at] = K.PNU21 * SDP[at] + K.PNU * adm[l];
        SZM[at] = K.PNU21 * SZP[at] + K.PNU * azm[l];
        STM[at] = K.PNU21 * STP[at] + K.PNU * atm[l];
        SQM[at] = K.PNU21 * SQP[at] + K.PNU * aqm[l];
      }
      real sdp = 2.0 * sdt[l] - adm[l];
      real stp = K.DELT2 * stt[l] + atm[l];
      real szp = K.DELT2 * SZT[at] + azm[l];
      real sqp = K.DELT2 * SQT[at] + aqm[l];
      SDT[at] = sdt[l];
      STT[at] = stt[l];
      SDP[at] = sdp;
      STP[at] = stp;
      SZP[at] = szp;
      SQP[at] = sqp;
      SD[at] = sdp;
      ST[at] = stp;
      SZ[at] = szp;
      SQ[at] = sqp;
    }
  }
}

// dynamics/wgsl/spectrald-diffusion.wgsl:1-60.
void spectrald_diffusion(Model& m) {
  const Consts& K = m.k;
  const int NL = m.NLEV, NR = m.NRSP;
  const real *sak = m.TB("sakpp"), *dampT = m.TB("damp"), *tdt = m.TB("tdisst"), *tdq = m.TB("tdissq"),
               *tdd = m.TB("tdissd"), *tdz = m.TB("tdissz"), *tfr = m.TB("tfrc"), *srp = m.TB("srp");
  real *SPP = m.F("spp"), *SZP = m.F("szp"), *STP = m.F("stp"), *SDP = m.F("sdp"), *SQP = m.F("sqp"),
         *SZT = m.F("szt"), *STT = m.F("stt"), *SDT = m.F("sdt"), *SQT = m.F("sqt"),
         *Z1 = m.F("zdsdp1"), *Z2 = m.F("zdszp1"), *Z3 = m.F("zdsdp2"), *Z4 = m.F("zdszp2");
  const real D2 = K.DELT2;
  for (int s = 0; s < NR; ++s) {
    if (s < 2) SPP[s] = 0.0;
    for (int l = 0; l < NL; ++l) {
      int at = l * NR + s;
      real szp = SZP[at] + D2 * SZT[at];
      real stp = STP[at] + D2 * STT[at];
      real sdp = SDP[at] + D2 * SDT[at];
      real sqp = SQP[at] + D2 * SQT[at];
      real sakpp = sak[at];
      real damp = dampT[l], tdisst = tdt[l], tdissq = tdq[l], tdissd = tdd[l], tdissz = tdz[l],
             tfrc = tfr[l];
      real stt = ((-damp - tdisst * sakpp) * stp + damp * srp[at]) / (1.0 + D2 * (damp + tdisst * sakpp));
      real sqt = -tdissq * sakpp * sqp / (1.0 + D2 * tdissq * sakpp);
      real zsdt1 = -tfrc * sdp / (1.0 + D2 * tfrc);
      real zsdt2 = -tdissd * sakpp * sdp / (1.0 + D2 * tdissd * sakpp);
      real zszt1 = -tfrc * szp / (1.0 + D2 * tfrc);
      real zszt2 = -tdissz * sakpp * szp / (1.0 + D2 * tdissz * sakpp);
      real szt = zszt1 + zszt2;
      if (s == 2) {
        zszt1 = zszt1 + K.PLAVOR * tfrc / (1.0 + D2 * tfrc);
        zszt2 = zszt2 + K.PLAVOR * tdissz * sakpp / (1.0 + D2 * tdissz * sakpp);
        szt = szt + K.PLAVOR * (tfrc / (1.0 + D2 * tfrc) + tdissz * sakpp / (1.0 + D2 * tdissz * sakpp));
      }
      SZP[at] = szp;
      STP[at] = stp;
      SDP[at] = sdp;
      SQP[at] = sqp;
      STT[at] = stt;
      SQT[at] = sqt;
      SDT[at] = zsdt1 + zsdt2;
      SZT[at] = szt;
      Z1[at] = zsdt1 * D2;
      Z2[at] = zszt1 * D2;
      Z3[at] = zsdt2 * D2;
      Z4[at] = zszt2 * D2;
    }
  }
}

// dynamics/wgsl/mkdheat.wgsl:1-44.
void mkdheat(Model& m, int stage) {
  const Consts& K = m.k;
  const int NH = m.NHOR;
  const real *ds = m.TB("dsigma"), *rcsq = m.TB("rcsq");
  real *DQ = m.F("dq"), *DP = m.F("dp"), *ZDEKIN = m.F("zdekin"), *ZDTDT = m.F("zdtdt"),
         *ZU = m.F("zu"), *ZV = m.F("zv"), *ZDU = m.F("zdu"), *ZDV = m.F("zdv");
  for (int i = 0; i < m.NLEV * NH; ++i) {
    int l = i / NH, h = i % NH;
    real heat = 1.0 + K.ADV * DQ[i];
    if (stage == 3) {
      real dp = DP[h];
      real dtdt = -ZDEKIN[i] * 0.5 / K.ACPD / heat / dp * K.GA / ds[l];
      ZDTDT[i] = dtdt / K.CT / K.WW;
      continue;
    }
    real scale = K.CV * std::sqrt(rcsq[h]);
    real u = ZU[i] * scale, v = ZV[i] * scale, du = ZDU[i] * scale, dv = ZDV[i] * scale;
    real change = du * (2.0 * u + du) + dv * (2.0 * v + dv);
    if (stage == 1) {
      real dtdt = -change / K.DELTSEC2 * 0.5 / K.ACPD / heat;
      ZDTDT[i] = dtdt / K.CT / K.WW;
    } else {
      ZDEKIN[i] = change / K.DELTSEC2 * DP[h] / K.GA * ds[l];
    }
  }
}

// dynamics/wgsl/mean-mode.wgsl:1-13.
void mean_mode(Model& m, const char* name) {
  real* t = m.F(name);
  for (int i = 0; i < m.NLEV * m.NRSP; ++i)
    if (i % m.NRSP != 0) t[i] = 0.0;
}

// dynamics/wgsl/spectrald-update.wgsl:1-45.
void spectrald_update(Model& m) {
  const Consts& K = m.k;
  const int NL = m.NLEV, NR = m.NRSP;
  bool filter = K.FILTER != 0;
  real *SPP = m.F("spp"), *SPM = m.F("spm"), *SP = m.F("sp"), *STT = m.F("stt"), *Z1 = m.F("zstt1"),
         *Z2 = m.F("zstt2"), *SZP = m.F("szp"), *STP = m.F("stp"), *SDP = m.F("sdp"), *SQP = m.F("sqp"),
         *SZT = m.F("szt"), *SDT = m.F("sdt"), *SQT = m.F("sqt"), *SZM = m.F("szm"), *STM = m.F("stm"),
         *SDM = m.F("sdm"), *SQM = m.F("sqm"), *SZ = m.F("sz"), *ST = m.F("st"), *SD = m.F("sd"),
         *SQ = m.F("sq");
  for (int s = 0; s < NR; ++s) {
    real spp = SPP[s];
    if (filter) SPM[s] = SPM[s] + K.PNU * spp;
    SP[s] = spp;
    for (int l = 0; l < NL; ++l) {
      int at = l * NR + s;
      real stt = STT[at] + Z1[at] + Z2[at];
      STT[at] = stt;
      real szp = SZP[at] + K.DELT2 * SZT[at];
      real stp = STP[at] + K.DELT2 * stt;
      real sdp = SDP[at] + K.DELT2 * SDT[at];
      real sqp = SQP[at] + K.DELT2 * SQT[at];
      SZP[at] = szp;
      STP[at] = stp;
      SDP[at] = sdp;
      SQP[at] = sqp;
      if (filter) {
        SZM[at] = SZM[at] + K.PNU * szp;
        STM[at] = STM[at] + K.PNU * stp;
        SDM[at] = SDM[at] + K.PNU * sdp;
        SQM[at] = SQM[at] + K.PNU * sqp;
      }
      SZ[at] = szp;
      ST[at] = stp;
      SD[at] = sdp;
      SQ[at] = sqp;
    }
  }
}

// dynamics/wgsl/physics-in.wgsl:1-34.
void physics_in(Model& m) {
  const Consts& K = m.k;
  const int NH = m.NHOR;
  const real *rcsq = m.TB("rcsq"), *t0 = m.TB("t0");
  real *GP = m.F("gp"), *DP = m.F("dp"), *DUDT = m.F("dudt"), *DVDT = m.F("dvdt"), *DTDT = m.F("dtdt"),
         *DQDT = m.F("dqdt"), *GUDT = m.F("gudt"), *GVDT = m.F("gvdt"), *GTDT = m.F("gtdt"),
         *GQDT = m.F("gqdt"), *DU = m.F("du"), *DV = m.F("dv"), *DT = m.F("dt"), *DQ = m.F("dq"),
         *GU = m.F("gu"), *GV = m.F("gv"), *GT = m.F("gt"), *GQ = m.F("gq");
  for (int h = 0; h < NH; ++h) {
    real dp = K.PSURF * std::exp(GP[h]);
    DP[h] = dp;
    real scale = std::sqrt(rcsq[h]);
    for (int l = 0; l < m.NLEP; ++l) {
      int at = l * NH + h;
      DUDT[at] = 0;
      DVDT[at] = 0;
      DTDT[at] = 0;
      DQDT[at] = 0;
      if (l < m.NLEV) {
        GUDT[at] = 0;
        GVDT[at] = 0;
        GTDT[at] = 0;
        GQDT[at] = 0;
        DU[at] = K.CV * GU[at] * scale;
        DV[at] = K.CV * GV[at] * scale;
        DT[at] = K.CT * (GT[at] + t0[l]);
        DQ[at] = GQ[at] * K.PSURF / dp;
      }
    }
  }
}

// dynamics/wgsl/physics-out.wgsl:1-21.
void physics_out(Model& m) {
  const Consts& K = m.k;
  const int NH = m.NHOR;
  const real* rcsq = m.TB("rcsq");
  real *GUDT = m.F("gudt"), *GVDT = m.F("gvdt"), *GTDT = m.F("gtdt"), *GQDT = m.F("gqdt"),
         *DUDT = m.F("dudt"), *DVDT = m.F("dvdt"), *DTDT = m.F("dtdt"), *DQDT = m.F("dqdt"), *DP = m.F("dp");
  for (int i = 0; i < m.NLEV * NH; ++i) {
    int h = i % NH;
    real scale = std::sqrt(rcsq[h]);
    GUDT[i] = DUDT[i] / scale / K.CV / K.WW + GUDT[i];
    GVDT[i] = DVDT[i] / scale / K.CV / K.WW + GVDT[i];
    GTDT[i] = DTDT[i] / K.CT / K.WW + GTDT[i];
    GQDT[i] = DQDT[i] * DP[h] / K.WW / K.PSURF + GQDT[i];
  }
}

// ----------------------------------------------------------------- fixer
// physics/fixer/wgsl/column.wgsl, row.wgsl, reduction/wgsl/sum.wgsl, apply.wgsl.
void fixer(Model& m) {
  const Consts& K = m.k;
  const int NH = m.NHOR, NL = m.NLEV;
  const real *ds = m.TB("dsigma"), *zgw = m.TB("zgw");
  real *DQ = m.F("dq"), *DP = m.F("dp"), *FIXQ = m.F("fixq"), *FNEG = m.F("fixneg"), *FPOS = m.F("fixpos"),
         *FSUM = m.F("fixsum"), *GQDT = m.F("gqdt");
  for (int h = 0; h < NH; ++h) {
    real negative = 0, positive = 0;
    for (int l = 0; l < NL; ++l) {
      real q = DQ[l * NH + h] * ds[l];
      if (DQ[l * NH + h] < 0) negative = negative + q;
      if (DQ[l * NH + h] > 0) positive = positive + q;
    }
    real zneg = -negative * DP[h] * zgw[h];
    real zpos = positive * DP[h] * zgw[h];
    real factor = 1.0;
    bool fixed = zneg > 0.0 && zpos >= zneg;
    if (fixed) {
      factor = (zpos - zneg) / zpos;
      zneg = 0;
      zpos = zpos * factor;
    }
    for (int l = 0; l < NL; ++l) {
      real q = DQ[l * NH + h];
      FIXQ[l * NH + h] = fixed ? std::max(q * factor, 0.0) : q;
    }
    FNEG[h] = zneg;
    FPOS[h] = zpos;
  }
  for (int row = 0; row < m.NLAT; ++row) {
    int first = row * m.NLON;
    real zneg = 0;
    for (int j = 0; j < m.NLON; ++j) zneg = zneg + FNEG[first + j];
    if (zneg <= 0) continue;
    real zpos = 0;
    for (int j = 0; j < m.NLON; ++j) zpos = zpos + FPOS[first + j];
    if (zpos < zneg) continue;
    real factor = (zpos - zneg) / zpos;
    for (int j = 0; j < m.NLON; ++j) {
      for (int l = 0; l < NL; ++l) {
        real& q = FIXQ[l * NH + first + j];
        q = std::max(q * factor, 0.0);
      }
      FNEG[first + j] = 0;
      FPOS[first + j] = FPOS[first + j] * factor;
    }
  }
  real a = 0, b = 0;
  for (int h = 0; h < NH; ++h) {
    a += FNEG[h];
    b += FPOS[h];
  }
  FSUM[0] = a;
  FSUM[1] = b;
  real zzneg = FSUM[0], zzpos = FSUM[1];
  for (int h = 0; h < NH; ++h) {
    real dp = DP[h];
    for (int l = 0; l < NL; ++l) {
      int at = l * NH + h;
      real q = FIXQ[at];
      if (zzneg > 0) q = std::max(q * ((zzpos - zzneg) / zzpos), 0.0);
      GQDT[at] = GQDT[at] + dp * (q - DQ[at]) / K.DELT2 / K.PSURF;
      DQ[at] = q;
    }
  }
}

// ----------------------------------------------------------------- surface flux
// physics/surface-flux/wgsl/surflx.wgsl:1-128.
void surflx(Model& m) {
  const Consts& K = m.k;
  const int NH = m.NHOR, low = m.NLEV - 1;
  const real dsigma = m.TB("dsigma")[low], zfac = m.TB("flux_sigfac")[0], zlnsig = m.TB("flux_lnsig")[0];
  real *DU = m.F("du"), *DV = m.F("dv"), *DT = m.F("dt"), *DQ = m.F("dq"), *DP = m.F("dp"),
         *DLS = m.F("dls"), *DZ0 = m.F("dz0"), *DTRANSH = m.F("dtransh"), *DTRANSM = m.F("dtransm"),
         *DUDT = m.F("dudt"), *DVDT = m.F("dvdt"), *DTDT = m.F("dtdt"), *DQDT = m.F("dqdt"),
         *DTAUX = m.F("dtaux"), *DTAUY = m.F("dtauy"), *DUST3 = m.F("dust3"), *DSHFL = m.F("dshfl"),
         *DSHDT = m.F("dshdt"), *DTSA = m.F("dtsa"), *DRHS = m.F("drhs"), *DWATC = m.F("dwatc"),
         *DEVAP = m.F("devap"), *DLHFL = m.F("dlhfl"), *DLHDT = m.F("dlhdt");
  const real VK = 0.4, moisture = 1.0 / K.RDBRV - 1.0;
  for (int h = 0; h < NH; ++h) {
    int lo = low * NH + h, sf = m.NLEV * NH + h;
    real u = DU[lo], v = DV[lo], t = DT[lo], q = DQ[lo], ts = DT[sf], qs = DQ[sf], dp = DP[h],
           dls = DLS[h];
    real dtsa = t * zfac * (1.0 + moisture * q);
    real zabsu2 = std::max(K.ZUMIN, u * u + v * v);
    real znl = -K.GASCON * 0.5 * (t + dtsa) * zlnsig / K.GA;
    real zbz0 = znl / DZ0[h];
    real zri = K.GA * znl / (zabsu2 * dtsa) * (dtsa - ts * (1.0 + moisture * qs));
    real zkblnz = VK / std::log(zbz0 + 1.0);
    real zkblnz2 = zkblnz * zkblnz;
    real zrifm, zrifh;
    if (zri <= 0.0) {
      real zdenom = 1.0 + 3.0 * K.VDIFF_C * K.VDIFF_B * std::sqrt(-1.0 * zri * (zbz0 + 1.0)) * zkblnz2;
      zrifm = 1.0 - 2.0 * K.VDIFF_B * zri / zdenom;
      if (dls < 1.0) {
        real zdth = -(dtsa - ts * (1.0 + moisture * qs));
        zrifh = std::pow(1.0 + std::pow(0.0016 * std::cbrt(zdth) / std::sqrt(zabsu2) / zkblnz2, 1.25), 0.8);
      } else {
        zrifh = 1.0 - 3.0 * K.VDIFF_B * zri / zdenom;
      }
    } else {
      real zdenom = std::sqrt(1.0 + K.VDIFF_D * zri);
      zrifh = 1.0 / (1.0 + 3.0 * K.VDIFF_B * zri * zdenom);
      zrifm = 1.0 / (1.0 + 2.0 * K.VDIFF_B * zri / zdenom);
    }
    real ztrans = std::sqrt(zabsu2) * zkblnz2;
    real transh = ztrans * zrifh, transm = ztrans * zrifm;
    DTRANSH[h] = transh;
    DTRANSM[h] = transm;
    real zkonst1 = K.GA * K.DELTSEC2 / (K.GASCON * dsigma);
    real zkonst2 = dsigma / K.DELTSEC2 / K.GA;
    real zkdiffm = zkonst1 * transm / ts;
    real zun = u / (1.0 + zkdiffm), zvn = v / (1.0 + zkdiffm);
    DUDT[lo] = DUDT[lo] + (zun - u) / K.DELTSEC2;
    DVDT[lo] = DVDT[lo] + (zvn - v) / K.DELTSEC2;
    real dtdt = DTDT[lo];
    if (K.NDHEAT != 0)
      dtdt = dtdt + -(zun * zun - u * u + zvn * zvn - v * v) / K.DELTSEC2 * 0.5 / K.ACPD / (1.0 + K.ADV * q);
    real taux = dp * zkonst2 * zkdiffm * zun, tauy = dp * zkonst2 * zkdiffm * zvn;
    DTAUX[h] = taux;
    DTAUY[h] = tauy;
    real ustar = std::sqrt(std::sqrt(taux * taux + tauy * tauy) * K.GASCON * ts / dp);
    DUST3[h] = ustar * ustar * ustar;
    real zkdiffh = zkonst1 * transh / ts;
    real ztn = (t + zkdiffh * ts) / (1.0 + zkdiffh * zfac);
    dtdt = dtdt + (ztn - t) / K.DELTSEC2;
    DTDT[lo] = dtdt;
    real moist = std::max(1.0, 1.0 + K.ADV * q);
    DSHFL[h] = zkonst2 * zkdiffh * dp * K.ACPD * moist * (ztn * zfac - ts);
    DSHDT[h] = -1.0 * zkonst2 * zkdiffh * dp * K.ACPD * moist;
    dtsa = ztn * zfac;
    DTSA[h] = dtsa;
    real zkdiffq = DRHS[h] * zkonst1 * transh / ts;
    real zqn = std::max(q, (q + zkdiffq * qs) / (1.0 + zkdiffq));
    if (dls > 0.0) zqn = std::min(zqn, DWATC[h] / K.DELTSEC * 1000.0 / dp / zkonst2 + q);
    DQDT[lo] = DQDT[lo] + (zqn - q) / K.DELTSEC2;
    real devap = -dp * zkonst2 / 1000.0 * (zqn - q);
    DEVAP[h] = devap;
    real latent = (ts > K.TMELT || dls < 0.5) ? K.ALV : K.ALS;
    real dlhfl = devap * latent * 1000.0;
    DLHFL[h] = dlhfl;
    real curvature = (ts - K.RA4) * (ts - K.RA4);
    real dlhdt = -1.0 * latent * zkdiffq * zkonst2 * dp * K.RA2 * (K.TMELT - K.RA4) * qs / curvature;
    DLHDT[h] = dlhfl == 0.0 ? 0.0 : dlhdt;
  }
}

// physics/diffusion/wgsl/implicit.wgsl:1-24 (diffuse).
static void diffuse(int NL, const real* ds, real* x, const real* k) {
  real ebs[MAXL];
  real ds0 = ds[0];
  ebs[0] = k[0] / (ds0 + k[0]);
  x[0] = ds0 * x[0] / (ds0 + k[0]);
  for (int l = 1; l < NL - 1; ++l) {
    real den = ds[l] + k[l] + k[l - 1] * (1.0 - ebs[l - 1]);
    ebs[l] = k[l] / den;
    x[l] = (x[l] * ds[l] + k[l - 1] * x[l - 1]) / den;
  }
  real dsn = ds[NL - 1];
  x[NL - 1] = (x[NL - 1] * dsn + k[NL - 2] * x[NL - 2]) / (dsn + k[NL - 2] * (1.0 - ebs[NL - 2]));
  for (int l = NL - 2; l >= 0; --l) x[l] = x[l] + ebs[l] * x[l + 1];
}

// physics/diffusion/wgsl/implicit.wgsl:26-47 (diffuse_potential).
static void diffuse_potential(int NL, const real* ds, real* x, const real* k, const real* skap) {
  real ebs[MAXL];
  real ds0 = ds[0];
  ebs[0] = k[0] / (ds0 + k[0] / skap[0]);
  x[0] = ds0 * x[0] / (ds0 + k[0] / skap[0]);
  for (int l = 1; l < NL - 1; ++l) {
    real den = ds[l] + (k[l] + k[l - 1] * (1.0 - ebs[l - 1] / skap[l - 1])) / skap[l];
    ebs[l] = k[l] / den;
    x[l] = (x[l] * ds[l] + k[l - 1] / skap[l - 1] * x[l - 1]) / den;
  }
  int last = NL - 1;
  real dsn = ds[last];
  x[last] = (x[last] * dsn + k[NL - 2] * x[NL - 2] / skap[NL - 2]) /
            (dsn + k[NL - 2] / skap[last] * (1.0 - ebs[NL - 2] / skap[NL - 2]));
  for (int l = NL - 2; l >= 0; --l) x[l] = x[l] + ebs[l] * x[l + 1] / skap[l + 1];
}

// physics/surface-flux/wgsl/vdiff.wgsl:1-120.
void vdiff(Model& m) {
  const Consts& K = m.k;
  const int NH = m.NHOR, NL = m.NLEV;
  const real *ds = m.TB("dsigma"), *sh = m.TB("sigmah"), *skapT = m.TB("vdiff_skap"),
               *skaphT = m.TB("vdiff_skaph"), *mixh2 = m.TB("vdiff_mixh2"), *mixm2 = m.TB("vdiff_mixm2"),
               *rdsg = m.TB("vdiff_rdsig"), *sh3 = m.TB("vdiff_sigmah3"), *kfac = m.TB("vdiff_kfac");
  real *DT = m.F("dt"), *DTDT = m.F("dtdt"), *DQ = m.F("dq"), *DQDT = m.F("dqdt"), *DU = m.F("du"),
         *DUDT = m.F("dudt"), *DV = m.F("dv"), *DVDT = m.F("dvdt");
  const real zkonst1 = K.GA * K.DELTSEC2 / K.GASCON;
  const real zkonst2 = zkonst1 * K.GA / K.GASCON;
  const real zkonst3 = zkonst2 * K.GA / K.GASCON;
  const real moisture = 1.0 / K.RDBRV - 1.0;
  for (int h = 0; h < NH; ++h) {
    real zt[MAXL], zq[MAXL], zu[MAXL], zv[MAXL], zabsu[MAXL], zskap[MAXL], zskaph[MAXL];
    for (int l = 0; l < NL; ++l) {
      int at = l * NH + h;
      zt[l] = DT[at] + DTDT[at] * K.DELTSEC2;
      zq[l] = DQ[at] + DQDT[at] * K.DELTSEC2;
      zu[l] = DU[at] + DUDT[at] * K.DELTSEC2;
      zv[l] = DV[at] + DVDT[at] * K.DELTSEC2;
      zabsu[l] = std::sqrt(zu[l] * zu[l] + zv[l] * zv[l]);
      zskap[l] = skapT[l];
      zskaph[l] = skaphT[l];
    }
    real kh[MAXL] = {0}, km[MAXL] = {0};
    for (int l = 0; l < NL - 1; ++l) {
      int lp = l + 1;
      real sigmah = sh[l], dsigma = ds[l], dsigmap = ds[lp];
      real zmixh2 = mixh2[l], zmixm2 = mixm2[l], zrdsig = rdsg[l], zfac = zkonst3 * sh3[l], zzkfac = kfac[l];
      real zrthl = (dsigmap + dsigma) / (zt[l] * dsigmap + zt[lp] * dsigma);
      real zdvds = std::max(K.ZUMIN, std::fabs(zabsu[l] - zabsu[lp])) * zrdsig;
      real zdthds = (zt[l] * (1.0 + moisture * zq[l]) / zskap[l] - zt[lp] * (1.0 + moisture * zq[lp]) / zskap[lp]) * zrdsig;
      real zri = zskaph[l] * K.GASCON * zdthds / (sigmah * zdvds * zdvds);
      real zrifh, zrifm;
      if (zri <= 0.0) {
        real dh = 1.0 + 3.0 * K.VDIFF_C * K.VDIFF_B * std::sqrt(-1.0 * zri) * zzkfac * zmixh2;
        real dm = 1.0 + 3.0 * K.VDIFF_C * K.VDIFF_B * std::sqrt(-1.0 * zri) * zzkfac * zmixm2;
        zrifh = 1.0 - 3.0 * K.VDIFF_B * zri / dh;
        zrifm = 1.0 - 2.0 * K.VDIFF_B * zri / dm;
      } else {
        real zdenom = std::sqrt(1.0 + K.VDIFF_D * zri);
        zrifh = 1.0 / (1.0 + 3.0 * K.VDIFF_B * zri * zdenom);
        zrifm = 1.0 / (1.0 + 2.0 * K.VDIFF_B * zri / zdenom);
      }
      kh[l] = zfac * zmixh2 * zrifh * zdvds * zrthl * zrthl * zrthl;
      km[l] = zfac * zmixm2 * zrifm * zdvds * zrthl * zrthl * zrthl;
    }
    real zun[MAXL], zvn[MAXL];
    for (int l = 0; l < NL; ++l) {
      zun[l] = zu[l];
      zvn[l] = zv[l];
    }
    diffuse(NL, ds, zun, km);
    diffuse(NL, ds, zvn, km);
    for (int l = 0; l < NL; ++l) {
      int at = l * NH + h;
      DUDT[at] = DUDT[at] + (zun[l] - zu[l]) / K.DELTSEC2;
      DVDT[at] = DVDT[at] + (zvn[l] - zv[l]) / K.DELTSEC2;
    }
    if (K.NDHEAT != 0) {
      real zke[MAXL], zken[MAXL];
      for (int l = 0; l < NL; ++l) zke[l] = zken[l] = 0.5 * zabsu[l] * zabsu[l];
      diffuse(NL, ds, zken, km);
      for (int l = 0; l < NL; ++l) {
        int at = l * NH + h;
        real zdtdt = -((zun[l] * zun[l] - zu[l] * zu[l] + zvn[l] * zvn[l] - zv[l] * zv[l]) / K.DELTSEC2 -
                         (zken[l] - zke[l]) / K.DELTSEC2) * 0.5 / K.ACPD / (1.0 + K.ADV * DQ[at]);
        DTDT[at] = DTDT[at] + zdtdt;
      }
    }
    real zqn[MAXL];
    for (int l = 0; l < NL; ++l) zqn[l] = zq[l];
    diffuse(NL, ds, zqn, kh);
    for (int l = 0; l < NL; ++l) DQDT[l * NH + h] = DQDT[l * NH + h] + (zqn[l] - zq[l]) / K.DELTSEC2;
    for (int l = 0; l < NL - 1; ++l) kh[l] = kh[l] * zskaph[l];
    real ztn[MAXL];
    for (int l = 0; l < NL; ++l) ztn[l] = zt[l];
    diffuse_potential(NL, ds, ztn, kh, zskap);
    for (int l = 0; l < NL; ++l) DTDT[l * NH + h] = DTDT[l * NH + h] + (ztn[l] - zt[l]) / K.DELTSEC2;
  }
}

// ----------------------------------------------------------------- radiation
constexpr real PI_ = 3.14159265359;
constexpr real TWOPI_ = PI_ + PI_;

// physics/radiation/wgsl/solang.wgsl:1-32.
void solang(Model& m) {
  const Consts& K = m.k;
  const real *sid = m.TB("sid"), *cola = m.TB("cola"), *RS = m.F("radiation_step");
  real* GMU0 = m.F("gmu0");
  for (int h = 0; h < m.NHOR; ++h) {
    int lat = h / m.NLON, lon = h % m.NLON;
    real hangle = RS[2] + lon * K.ZRLON - PI_;
    if (hangle < -PI_) hangle = hangle + TWOPI_;
    if (hangle > PI_) hangle = hangle - TWOPI_;
    if (K.NFIXED == 1) hangle = hangle + PI_;
    real muz = RS[0] * sid[lat] + cola[lat] * RS[1] * std::cos(hangle);
    GMU0[h] = muz > K.ZDAWN ? muz : 0.0;
  }
}

// physics/radiation/wgsl/mko3.wgsl:1-37.
void mko3(Model& m) {
  const Consts& K = m.k;
  const int NH = m.NHOR;
  const real *sidT = m.TB("sid"), *lnsig = m.TB("rad_lnsig"), *ds = m.TB("dsigma"), *RS = m.F("radiation_step");
  real *DP = m.F("dp"), *DT = m.F("dt"), *DQO3 = m.F("dqo3");
  const real ZFO3 = 100.0 / 2.14;
  for (int h = 0; h < NH; ++h) {
    real sid = sidT[h / m.NLON];
    real za = K.A0O3 + K.A1O3 * std::fabs(sid) + K.ACO3 * sid * RS[4];
    real dp = DP[h];
    real o3t = za, zh = 0.0;
    for (int l = m.NLEV - 1; l >= 1; --l) {
      zh = zh - DT[l * NH + h] * K.GASCON / K.GA * lnsig[l];
      real o3 = -(za + za * K.ZCONST) / (1.0 + std::exp((zh - K.BO3) / K.CO3)) + o3t;
      DQO3[l * NH + h] = o3 * K.GA / (ZFO3 * ds[l] * dp);
      o3t = o3t - o3;
    }
    DQO3[h] = o3t * K.GA / (ZFO3 * ds[0] * dp);
  }
}

static real fpow(real x, real y) { return x == 0.0 ? 0.0 : std::exp(y * std::log(x)); }

// physics/radiation/wgsl/swr.wgsl:1-276.
void swr(Model& m) {
  const Consts& K = m.k;
  const int NH = m.NHOR, NL = m.NLEV;
  const real *ds = m.TB("dsigma"), *sg = m.TB("sigma"), *RS = m.F("radiation_step");
  real *GMU0 = m.F("gmu0"), *DFU = m.F("dfu"), *DFD = m.F("dfd"), *DSWFL = m.F("dswfl"), *DP = m.F("dp"),
         *DCC = m.F("dcc"), *DQL = m.F("dql"), *DQO3 = m.F("dqo3"), *DQ = m.F("dq"), *DT = m.F("dt"),
         *DALB = m.F("dalb"), *DSALB = m.F("dsalb"), *DLS = m.F("dls"), *DICEC = m.F("dicec");
  const real ZERO = 1.0e-6, ZBETTA = 1.66, ZMBAR = 1.9, ZFO3 = 100.0 / 2.14, ZMU00 = 0.5,
               INV_LN10 = 0.43429448190325176;
  auto ozone = [&](real o3) {
    return (0.02118 * o3 / (1.0 + 0.042 * o3 + 0.000323 * (o3 * o3)) + 1.082 * o3 / fpow(1.0 + 138.6 * o3, 0.805) +
            0.0658 * o3 / (1.0 + (103.6 * o3) * (103.6 * o3) * (103.6 * o3))) / K.ZSOLAR1;
  };
  auto vapour = [&](real wv) { return 2.9 * wv / (fpow(1.0 + 141.5 * wv, 0.635) + 5.925 * wv) / K.ZSOLAR2; };
  for (int h = 0; h < NH; ++h) {
    real mu0 = GMU0[h], gdist2 = RS[3];
    real ftop1 = K.ZSOLAR1 * K.GSOL0 * gdist2 * mu0;
    real ftop2 = K.ZSOLAR2 * K.GSOL0 * gdist2 * mu0;
    if (!(ftop1 + ftop2 > ZERO)) {
      for (int l = 0; l < m.NLEP; ++l) {
        DFU[l * NH + h] = 0;
        DFD[l * NH + h] = 0;
        DSWFL[l * NH + h] = 0;
      }
      continue;
    }
    real dp = DP[h];
    real rcl1[MAXL], rcl1s[MAXL], rcl2[MAXL], rcl2s[MAXL], tcl2[MAXL], tcl2s[MAXL];
    real cs = 1.0;
    for (int l = 0; l < NL; ++l) {
      real cc = DCC[l * NH + h];
      rcl1[l] = rcl1s[l] = rcl2[l] = rcl2s[l] = 0;
      tcl2[l] = tcl2s[l] = 1;
      if (cc > 0) {
        real lwp = std::min(1000.0, 1000.0 * DQL[l * NH + h] * dp / K.GA * ds[l]);
        real tau = 2.0 * fpow(std::log(lwp + 1.5) * INV_LN10, 3.9);
        real zlog = std::log(1000.0 / tau);
        real b2 = K.ZB4 / std::log(3.0 + 0.1 * tau);
        real om0 = std::min(0.9999, 1.0 - K.ZB5 * zlog);
        real un = 1.0 - om0, uz = un + 2.0 * b2 * om0, u = std::sqrt(uz / un);
        real ex = std::exp(std::min(25.0, tau * std::sqrt(uz * un) / ZMU00));
        real r = (u + 1.0) * (u + 1.0) * ex - (u - 1.0) * (u - 1.0) / ex;
        rcl1s[l] = 1.0 - 1.0 / (1.0 + K.ZB3 * tau);
        tcl2s[l] = 4.0 * u / r;
        rcl2s[l] = (u * u - 1.0) / r * (ex - 1.0 / ex);
        real b1 = K.TSWR1 * std::sqrt(mu0);
        b2 = K.TSWR2 * std::sqrt(mu0) / std::log(3.0 + 0.1 * tau);
        om0 = std::min(0.9999, 1.0 - K.TSWR3 * mu0 * mu0 * zlog);
        un = 1.0 - om0;
        uz = un + 2.0 * b2 * om0;
        u = std::sqrt(uz / un);
        ex = std::exp(std::min(25.0, tau * std::sqrt(uz * un) / mu0));
        r = (u + 1.0) * (u + 1.0) * ex - (u - 1.0) * (u - 1.0) / ex;
        real direct1 = 1.0 - 1.0 / (1.0 + b1 * tau / mu0);
        real directT = 4.0 * u / r;
        real direct2 = (u * u - 1.0) / r * (ex - 1.0 / ex);
        rcl1[l] = cs * direct1 + (1.0 - cs) * rcl1s[l];
        tcl2[l] = cs * directT + (1.0 - cs) * tcl2s[l];
        rcl2[l] = cs * direct2 + (1.0 - cs) * rcl2s[l];
      }
      cs = cs * (1.0 - cc);
    }
    real zm = 35.0 / std::sqrt(1.0 + 1224.0 * mu0 * mu0);
    real o3l[MAXL], xo3l[MAXL], wvl[MAXL], ywvl[MAXL];
    real o3t = 0, xo3t = 0, wvt = 0, ywvt = 0;
    cs = 1.0;
    for (int l = 0; l < NL; ++l) {
      real dsigma = ds[l];
      real o3 = ZFO3 * dsigma * dp * DQO3[l * NH + h] / K.GA;
      o3t = o3t + o3;
      xo3t = cs * (xo3t + zm * o3) + (1.0 - cs) * (xo3t + ZMBAR * o3);
      o3l[l] = o3t;
      xo3l[l] = xo3t;
      real wv = 0.1 * dsigma * DQ[l * NH + h] * dp / K.GA * std::sqrt(273.0 / DT[l * NH + h]) * sg[l] * dp / 100000.0;
      wvt = wvt + wv;
      ywvt = cs * (ywvt + zm * wv) + (1.0 - cs) * (ywvt + ZBETTA * wv);
      wvl[l] = wvt;
      ywvl[l] = ywvt;
      cs = cs * (1.0 - DCC[l * NH + h]);
    }
    real ta1 = 1, ta1s = 1, ra1 = 0, ra1s = 0, ta2 = 1, ta2s = 1, ra2 = 0, ra2s = 0;
    real to3t = 1.0, to3tu = 1.0 - ozone(xo3t + ZMBAR * o3t);
    real twvt = 1.0, twvtu = 1.0 - vapour(ywvt + ZBETTA * wvt);
    real ccn = DCC[(NL - 1) * NH + h];
    real scf = K.RCOEFF * dp / 101100.0 * 9.80665 / K.GA;
    real diffuseRayleigh = 1.0 - std::exp(scf * K.LN_DIFFUSE_RAYLEIGH);
    real rcsuSurface = diffuseRayleigh * (1.0 - ccn);
    real rcsSurface = (1.0 - std::exp(scf * std::log(1.0 - 0.219 / (1.0 + 0.816 * mu0)))) * cs +
                        diffuseRayleigh * (1.0 - cs - ccn);
    real t1[MAXL + 1], t2[MAXL + 1], r1s[MAXL + 1], r2s[MAXL + 1];
    real tb1[MAXL], tb1u[MAXL], rb1[MAXL], rb1s[MAXL], tb2[MAXL], tb2u[MAXL], rb2[MAXL], rb2s[MAXL];
    for (int l = 0; l < NL; ++l) {
      real cc = DCC[l * NH + h];
      t1[l] = ta1;
      t2[l] = ta2;
      r1s[l] = ra1s;
      r2s[l] = ra2s;
      bool surface = l == NL - 1;
      rb1[l] = (surface ? rcsSurface : 0.0) + rcl1[l] * cc;
      rb1s[l] = (surface ? rcsuSurface : 0.0) + rcl1s[l] * cc;
      real o3 = xo3l[l];
      real to3 = (1.0 - ozone(o3)) / to3t;
      to3t = to3t * to3;
      o3 = xo3t + ZMBAR * (o3t - o3l[l]);
      real to3u = to3tu / (1.0 - ozone(o3));
      to3tu = to3tu / to3u;
      tb1[l] = 1.0 - (1.0 - to3) * (1.0 - cc) - rb1[l];
      tb1u[l] = 1.0 - (1.0 - to3u) * (1.0 - cc) - rb1s[l];
      real m1 = 1.0 / (1.0 - ra1s * rb1s[l]);
      ra1 = ra1 + ta1 * rb1[l] * ta1s * m1;
      ta1 = ta1 * tb1[l] * m1;
      ra1s = rb1s[l] + tb1u[l] * ra1s * tb1[l] * m1;
      ta1s = tb1u[l] * ta1s * m1;
      rb2[l] = rcl2[l] * cc;
      rb2s[l] = rcl2s[l] * cc;
      real wv = ywvl[l];
      real twv = (1.0 - vapour(wv)) / twvt;
      twvt = twvt * twv;
      wv = ywvt + ZBETTA * (wvt - wvl[l]);
      real twvu = twvtu / (1.0 - vapour(wv));
      twvtu = twvtu / twvu;
      tb2[l] = 1.0 - (1.0 - twv) * (1.0 - cc) - (1.0 - tcl2[l]) * cc;
      tb2u[l] = 1.0 - (1.0 - twvu) * (1.0 - cc) - (1.0 - tcl2s[l]) * cc;
      real m2 = 1.0 / (1.0 - ra2s * rb2s[l]);
      ra2 = ra2 + ta2 * rb2[l] * ta2s * m2;
      ta2 = ta2 * tb2[l] * m2;
      ra2s = rb2s[l] + tb2u[l] * ra2s * tb2[l] * m2;
      ta2s = tb2u[l] * ta2s * m2;
    }
    t1[NL] = ta1;
    t2[NL] = ta2;
    r1s[NL] = ra1s;
    r2s[NL] = ra2s;
    bool star = K.NSTARTEMP != 0;
    real dalb = DALB[h], salb1 = DSALB[h], salb2 = DSALB[NH + h];
    ra1s = star ? salb1 : dalb;
    ra2s = star ? salb2 : dalb;
    real dls = DLS[h], dicec = DICEC[h];
    real water = (1.0 - dls) * (1.0 - dicec) * std::min(0.05 / (mu0 + 0.15), 0.15);
    real nalb1 = dls * salb1 + (1.0 - dls) * dicec * salb1 + water;
    real nalb2 = dls * salb2 + (1.0 - dls) * dicec * salb2 + water;
    DSALB[h] = nalb1;
    DSALB[NH + h] = nalb2;
    real albedo = star ? K.ZSOLARS1 * nalb1 + K.ZSOLARS2 * nalb2 : dls * dalb + (1.0 - dls) * dicec * dalb + water;
    DALB[h] = albedo;
    ra1 = star ? nalb1 : albedo;
    ra2 = star ? nalb2 : albedo;
    real rl1[MAXL + 1], rl2[MAXL + 1], rl1s[MAXL + 1], rl2s[MAXL + 1];
    for (int l = NL - 1; l >= 0; --l) {
      rl1[l + 1] = ra1;
      rl2[l + 1] = ra2;
      rl1s[l + 1] = ra1s;
      rl2s[l + 1] = ra2s;
      real d1 = 1.0 - ra1s * rb1s[l];
      ra1 = rb1[l] + tb1[l] * ra1 * tb1u[l] / d1;
      ra1s = rb1s[l] + tb1u[l] * ra1s * tb1u[l] / d1;
      real d2 = 1.0 - ra2s * rb2s[l];
      ra2 = rb2[l] + tb2[l] * ra2 * tb2u[l] / d2;
      ra2s = rb2s[l] + tb2u[l] * ra2s * tb2u[l] / d2;
    }
    rl1[0] = ra1;
    rl2[0] = ra2;
    rl1s[0] = ra1s;
    rl2s[0] = ra2s;
    for (int l = 0; l < m.NLEP; ++l) {
      real m1 = 1.0 / (1.0 - r1s[l] * rl1s[l]);
      real m2 = 1.0 / (1.0 - r2s[l] * rl2s[l]);
      real fu = -t1[l] * rl1[l] * m1 * ftop1 + -t2[l] * rl2[l] * m2 * ftop2;
      real fd = t1[l] * m1 * ftop1 + t2[l] * m2 * ftop2;
      DFU[l * NH + h] = fu;
      DFD[l * NH + h] = fd;
      DSWFL[l * NH + h] = fu + fd;
    }
  }
}

// physics/radiation/wgsl/lwr.wgsl:1-179.
void lwr(Model& m) {
  const Consts& K = m.k;
  const int NH = m.NHOR, NL = m.NLEV, NP = m.NLEP;
  const real *sg = m.TB("sigma"), *sh = m.TB("sigmah"), *zzf1 = m.TB("lwr_zzf1"), *zzf3 = m.TB("lwr_zzf3");
  real *DP = m.F("dp"), *DT = m.F("dt"), *DLS = m.F("dls"), *DQ = m.F("dq"), *DQO3 = m.F("dqo3"),
         *DQCO2 = m.F("dqco2"), *DCC = m.F("dcc"), *DQL = m.F("dql"), *DFTU = m.F("dftu"), *DFTD = m.F("dftd"),
         *DLWFL = m.F("dlwfl");
  const real ZERO = 1.0e-6, ZFH2O = 0.1, ZFO3 = 100.0 / 2.14;
  for (int h = 0; h < NH; ++h) {
    real dp = DP[h], ps2 = dp * dp;
    real st4[MAXL + 1], st4h[MAXL + 1];
    for (int l = 0; l < NP; ++l) {
      real t = DT[l * NH + h], t2 = t * t;
      st4[l] = K.SBK * (t2 * t2);
    }
    st4h[0] = st4[0] - (st4[0] - st4[1]) * sg[0] / (sg[0] - sg[1]);
    for (int l = 1; l < NL; ++l) {
      real above = sg[l - 1], half = sh[l - 1], level = sg[l];
      st4h[l] = (st4[l] * (above - half) + st4[l - 1] * (half - level)) / (above - level);
    }
    int n = NL - 1;
    if ((st4[n] - st4h[n]) * (st4[n] - st4[NL]) > 0.0) {
      st4h[NL] = st4[NL];
    } else {
      real sn = sg[n], sm = sg[n - 1];
      st4h[NL] = st4[n] + (st4[n] - st4[n - 1]) * (1.0 - sn) / (sn - sm);
    }
    real bu[MAXL + 2], bd[MAXL + 2];
    bd[0] = 0.0;
    real dls = DLS[h];
    real eps = dls + 0.98 * (1.0 - dls);
    bu[NP] = eps * st4[NL];
    real q[MAXL], qo3[MAXL], qco2[MAXL], taucc0[MAXL];
    for (int l = 0; l < NL; ++l) {
      real sfac = zzf1[l] * ps2;
      q[l] = ZFH2O * sfac * DQ[l * NH + h];
      qo3[l] = ZFO3 * sfac * DQO3[l * NH + h];
      qco2[l] = K.ZFCO2_ZZF2 * sfac * DQCO2[l * NH + h];
      taucc0[l] = 1.0 - DCC[l * NH + h] * (1.0 - std::exp(zzf3[l] * DQL[l * NH + h] * dp));
    }
    real dftu[MAXL + 1] = {0}, dftd[MAXL + 1] = {0};
    real taucs[MAXL], tau[MAXL], tausf[MAXL];
    for (int j = 0; j < NL; ++j) {
      real taucc = 1.0, sumwv = 0, sumo3 = 0, sumco2 = 0;
      for (int kk = j; kk < NL; ++kk) {
        sumwv = sumwv + q[kk];
        sumo3 = sumo3 + qo3[kk];
        sumco2 = sumco2 + qco2[kk];
        real ah2o = sumwv <= 0.01 ? 0.846 * fpow(sumwv + 3.59e-5, 0.243) - K.ZH2O0A
                                    : 0.24 * std::log10(sumwv + 0.01) + K.ZAH2OC;
        if (K.TH2OC > 0.0) ah2o = std::min(ah2o + (1.0 - std::exp(-K.TH2OC * sumwv)), 1.0);
        real aco2 = sumco2 <= 1.0 ? 0.0676 * fpow(sumco2 + 0.01022, 0.421) - K.ZCO20
                                    : 0.0546 * std::log10(sumco2) + K.ZACO2C;
        real th2o = sumwv <= 2.0 ? 1.0 - (0.832 * fpow(sumwv + 0.0286, 0.26) - K.ZH2O0)
                                   : std::max(0.0, K.ZTH2OC - 0.1196 * std::log(sumwv - 0.6931));
        real ao3 = sumo3 <= 0.01 ? 0.209 * fpow(sumo3 + 7.0e-5, 0.436) - K.ZAO30
                                   : 0.0212 * std::log10(sumo3) + K.ZAO3C;
        real cs = std::min(1.0 - ZERO, std::max(ZERO, 1.0 - ah2o - ao3 - aco2 * th2o));
        taucs[kk] = cs;
        taucc = taucc * taucc0[kk];
        tau[kk] = cs * taucc;
      }
      if (j == 0) {
        real tau0 = 1.0 - ZERO;
        for (int kk = 0; kk < NL; ++kk) {
          tau0 = taucs[kk] / tau0 * taucc0[kk] * K.TPOFMT;
          tau0 = std::min(1.0 - ZERO, std::max(ZERO, tau0));
          if ((st4[kk] - st4h[kk]) * (st4[kk] - st4h[kk + 1]) > 0.0) {
            bd[kk + 1] = 0.5 * st4[kk] + 0.25 * (st4h[kk] + st4h[kk + 1]);
            bu[kk + 1] = bd[kk + 1];
          } else {
            bd[kk + 1] = (st4h[kk + 1] - tau0 * st4h[kk]) / (1.0 - tau0) - (st4h[kk] - st4h[kk + 1]) / std::log(tau0);
            bu[kk + 1] = st4h[kk] + st4h[kk + 1] - bd[kk + 1];
          }
          tau0 = taucs[kk];
        }
      }
      dftu[j] = dftu[j] - bu[j + 1];
      dftd[j] = dftd[j] + bd[j];
      real bdl = bd[j] - bd[j + 1];
      for (int kk = j; kk < NL; ++kk) {
        dftu[j] = dftu[j] - (bu[kk + 2] - bu[kk + 1]) * tau[kk];
        dftd[kk + 1] = dftd[kk + 1] + bdl * tau[kk];
      }
      tausf[j] = tau[NL - 1];
    }
    dftu[NL] = dftu[NL] - bu[NP];
    dftd[NL] = dftd[NL] + bd[NL];
    real reflected = (1.0 - eps) * dftd[NL];
    for (int l = 0; l < NL; ++l) dftu[l] = dftu[l] - tausf[l] * reflected;
    for (int l = 0; l < NP; ++l) {
      DFTU[l * NH + h] = dftu[l];
      DFTD[l * NH + h] = dftd[l];
      DLWFL[l * NH + h] = dftu[l] + dftd[l];
    }
  }
}

// physics/radiation/wgsl/radstep.wgsl:1-32.
void radstep(Model& m) {
  const Consts& K = m.k;
  const int NH = m.NHOR;
  const real *lnsig = m.TB("rad_lnsig"), *ds = m.TB("dsigma");
  real *DFLUX = m.F("dflux"), *DLWFL = m.F("dlwfl"), *DSWFL = m.F("dswfl"), *DP = m.F("dp"), *DT = m.F("dt"),
         *DQ = m.F("dq"), *DTDT = m.F("dtdt"), *DTDTSWR = m.F("dtdtswr"), *DTDTLWR = m.F("dtdtlwr"),
         *DCONV = m.F("dconv");
  for (int h = 0; h < NH; ++h) {
    for (int l = 0; l < m.NLEP; ++l) DFLUX[l * NH + h] = DLWFL[l * NH + h] + DSWFL[l * NH + h];
    real dp = DP[h];
    for (int l = 0; l < m.NLEV; ++l) {
      int at = l * NH + h, bl = (l + 1) * NH + h;
      real zdh = -DT[at] * K.GASCON / K.GA * lnsig[l];
      real den = ds[l] * dp * K.ACPD * (1.0 + K.ADV * DQ[at]);
      real flux = DFLUX[at], below = DFLUX[bl];
      DTDT[at] = DTDT[at] - K.GA * (below - flux) / den;
      DTDTSWR[at] = -K.GA * (DSWFL[bl] - DSWFL[at]) / den;
      DTDTLWR[at] = -K.GA * (DLWFL[bl] - DLWFL[at]) / den;
      DCONV[at] = (flux - below) / (zdh + 1.0e-9);
    }
  }
}

// ----------------------------------------------------------------- precipitation
struct Parcel {
  real t, q, cor;
  bool saturated;
};

static real sat_capped(const Consts& K, real t, real p) {
  return std::min(K.RDBRV * K.RA1 * std::exp(K.RA2 * (t - K.TMELT) / (t - K.RA4)) / p, K.RDBRV);
}
static real sat_divided(const Consts& K, real t, real p) {
  real q = sat_capped(K, t, p);
  return q / (1.0 - K.MOIST * q);
}

// physics/precipitation/wgsl/kuo.wgsl:20-43 (condense).
static Parcel condense(const Consts& K, real t0, real q0, real p) {
  real s = sat_capped(K, t0, p);
  real cor = 1.0 / (1.0 - K.MOIST * s);
  s = s * cor;
  if (!(s < q0)) return {t0, q0, cor, false};
  real t = t0, q = q0;
  real lcp = (t0 < K.TMELT ? K.ALS : K.ALV) / (K.ACPD * (1.0 + K.ADV * q0));
  for (int i = 0; i < 2; ++i) {
    if (i == 1) {
      s = sat_capped(K, t, p);
      cor = 1.0 / (1.0 - K.MOIST * s);
      s = s * cor;
    }
    real dqsdt = K.RA2 * (K.TMELT - K.RA4) * s * cor / ((t - K.RA4) * (t - K.RA4));
    real rain = (q - s) / (1.0 + lcp * dqsdt);
    t = t + lcp * rain;
    q = q - rain;
  }
  return {t, q, cor, true};
}

static real powi(real x, int n) {
  real base = x;
  unsigned mm = (unsigned)std::abs(n);
  real result = (mm & 1u) ? x : 1.0;
  mm >>= 1;
  while (mm) {
    base = base * base;
    if (mm & 1u) result = result * base;
    mm >>= 1;
  }
  return n < 0 ? 1.0 / result : result;
}

// physics/precipitation/wgsl/kuo.wgsl:45-298 (mkdqtgp, kuo, mkshallow).
void kuo(Model& m) {
  const Consts& K = m.k;
  const int NH = m.NHOR, NL = m.NLEV, NM = m.NLEM;
  const real *ds = m.TB("dsigma"), *sg = m.TB("sigma"), *sh = m.TB("sigmah"), *skapT = m.TB("vdiff_skap"),
               *skaph = m.TB("vdiff_skaph"), *vrd = m.TB("vdiff_rdsig"), *zfacT = m.TB("kuo_zfac");
  real *DP = m.F("dp"), *DQT = m.F("dqt"), *DQ = m.F("dq"), *DQDT = m.F("dqdt"), *DT = m.F("dt"),
         *DTDT = m.F("dtdt"), *DPRCL = m.F("dprcl"), *DPRSCL = m.F("dprscl"), *ICCLEV = m.F("icclev"),
         *ICCTOT = m.F("icctot");
  for (int h = 0; h < NH; ++h) {
    real dp = DP[h];
    real zdqt[MAXL], zqe[MAXL], zte[MAXL], zdqtot[MAXL], zalcpe[MAXL], zacpe[MAXL], zdqdt[MAXL], zdtdt[MAXL];
    for (int l = 0; l < NL; ++l) {
      int at = l * NH + h;
      zdqt[l] = DQT[at] * K.PSURF * K.WW / dp;
      DQT[at] = zdqt[l];
      real dq = DQ[at], dqdt = DQDT[at];
      zdqtot[l] = (zdqt[l] + dqdt) * K.DELTSEC2;
      zqe[l] = dq + dqdt * K.DELTSEC2;
      zte[l] = DT[at] + DTDT[at] * K.DELTSEC2;
      zacpe[l] = K.ACPD * (1.0 + K.ADV * dq);
      zalcpe[l] = K.ALV / zacpe[l];
      zdqdt[l] = 0;
      zdtdt[l] = 0;
    }
    int ilift = -1, itop = -1;
    real zi = 0, zpt = 0, zpq = 0, zbeta = 0, zpbeta = 0, ztp = 0, zqp = 0;
    int n = NL - 1;
    real dsn = ds[n];
    real ztsurf = DT[NL * NH + h] * skapT[n];
    if (zdqtot[n] > 0.0 && ztsurf > zte[n]) {
      real p = dp * sg[n];
      real zqsnl = sat_divided(K, zte[n], p);
      real zqnew = DQ[NL * NH + h] * std::min(1.0, zqe[n] / zqsnl);
      Parcel parcel = condense(K, ztsurf, zqnew, p);
      if (parcel.saturated) {
        ilift = m.NLEP;
        itop = NL;
        ztp = parcel.t;
        zqp = parcel.q;
        real zqsa = sat_divided(K, zte[n], p);
        zdqdt[n] = std::max(zqsa - zqe[n], 0.0);
        zdtdt[n] = ztp - zte[n];
        zpt = zdtdt[n] * dsn * zacpe[n];
        zpq = zdqdt[n] * dsn * K.ALV;
        zbeta = std::min(1.0, zqe[n] / zqsa) * dsn;
        zpbeta = dsn;
        zi = zdqtot[n] * dsn * K.ALV;
      }
    }
    for (int l = NM - 1; l >= 0; --l) {
      int lu = l, lp = l + 1;
      if (ilift == -1 && zdqtot[lp] > 0.0) {
        real p = dp * sg[lu];
        Parcel parcel = condense(K, zte[lp] * zfacT[lu], zqe[lp], p);
        if (parcel.saturated && parcel.t > zte[lu]) {
          real dsl = ds[lu], dsp = ds[lp];
          ilift = l + 2;
          itop = l + 1;
          ztp = parcel.t;
          zqp = parcel.q;
          real zqsa = sat_divided(K, zte[lu], p);
          zdqdt[lu] = std::max(zqsa - zqe[lu], 0.0);
          zdtdt[lu] = ztp - zte[lu];
          zpt = zdtdt[lu] * dsl * zacpe[lu];
          zpq = zdqdt[lu] * dsl * K.ALV;
          zbeta = std::min(1.0, zqe[lu] / zqsa) * dsl;
          zpbeta = dsl;
          real pp = dp * sg[lp];
          real zqsnl = sat_divided(K, zte[lp], pp);
          if (zqe[lp] > zqsnl) {
            real t = zte[lp], q = zqe[lp];
            real lcp = (t < K.TMELT ? K.ALS : K.ALV) / (K.ACPD * (1.0 + K.ADV * q));
            real cor = parcel.cor;
            for (int i = 0; i < 2; ++i) {
              if (i == 1) {
                zqsnl = sat_capped(K, t, pp);
                cor = 1.0 / (1.0 - K.MOIST * zqsnl);
                zqsnl = zqsnl * cor;
              }
              real dqsdt = K.RA2 * (K.TMELT - K.RA4) * zqsnl * cor / ((t - K.RA4) * (t - K.RA4));
              real rain = (q - zqsnl) / (1.0 + lcp * dqsdt);
              t = t + lcp * rain;
              q = q - rain;
            }
            zdqdt[lp] = std::max(q - zqe[lp], 0.0);
            zdtdt[lp] = t - zte[lp];
            zpt = zdtdt[lp] * dsp * zacpe[lp] + zpt;
            zpq = zdqdt[lp] * dsp * K.ALV + zpq;
            zbeta = std::min(1.0, zqe[lp] / zqsnl) * dsp + zbeta;
            zpbeta = dsp + zpbeta;
          }
          zi = zdqtot[lu] * dsl * K.ALV + zdqtot[lp] * dsp * K.ALV;
        }
      }
    }
    for (int l = NM - 1; l >= 0; --l) {
      int lu = l;
      if (itop == l + 2) {
        real p = dp * sg[lu];
        Parcel parcel = condense(K, ztp * zfacT[lu], zqp, p);
        if (parcel.saturated && parcel.t > zte[lu]) {
          real dsl = ds[lu];
          itop = l + 1;
          ztp = parcel.t;
          zqp = parcel.q;
          real zqsa = sat_divided(K, zte[lu], p);
          zdqdt[lu] = std::max(zqsa - zqe[lu], 0.0);
          zdtdt[lu] = ztp - zte[lu];
          zpt = zdtdt[lu] * dsl * zacpe[lu] + zpt;
          zpq = zdqdt[lu] * dsl * K.ALV + zpq;
          zbeta = std::min(1.0, zqe[lu] / zqsa) * dsl + zbeta;
          zpbeta = zpbeta + dsl;
          zi = zdqtot[lu] * dsl * K.ALV + zi;
        }
      }
    }
    zi = std::max(0.0, zi);
    real zrhm = zpbeta > 0.0 ? zbeta / zpbeta : 0.0;
    real beta = 1.0;
    if (zrhm >= K.RHBETA) beta = powi((1.0 - zrhm) / (1.0 - K.RHBETA), (int)K.NBETA);
    real zat = zpt > 0.0 ? zi * (1.0 - beta) / zpt : 0.0;
    real zaq = zpq > 0.0 ? zi * beta / zpq : 0.0;
    bool shallow = itop > 0 && (dp * sg[itop - 1] > K.PDEEP || zi <= 0.0);
    real icctot = 0;
    for (int l = 0; l < NL; ++l) {
      int level = l + 1, at = l * NH + h;
      real dprcl = 0, icclev = 0;
      if (ilift >= level && itop <= level && zi > 0.0 && !shallow) {
        DQDT[at] = zaq * zdqdt[l] / K.DELTSEC2 - zdqt[l];
        DTDT[at] = zat * zdtdt[l] / K.DELTSEC2 + DTDT[at];
        dprcl = zat * zdtdt[l] * ds[l] / zalcpe[l] / K.DELTSEC2;
      }
      if (dprcl > 0.0) {
        icclev = 1.0;
        icctot = icctot + 1.0;
      }
      if (sg[l] < 0.4 && icclev == 1.0 && itop == level) icclev = 2.0;
      DPRCL[at] = dprcl;
      DPRSCL[at] = 0;
      ICCLEV[at] = icclev;
    }
    ICCTOT[h] = icctot;
    if (!shallow) continue;
    real zkonst1 = K.GA * K.DELTSEC2 / K.GASCON;
    real zkonst2 = K.RKSHALLOW * zkonst1 * K.GA / K.GASCON;
    int kktop = 1;
    for (int level = 2; level <= NM; ++level)
      if (dp * sg[level - 1] < K.PDEEPTH) kktop = level;
    int ktop = std::max(itop, kktop);
    real zkdiff[MAXL] = {0}, skap[MAXL];
    for (int l = 0; l < NL; ++l) skap[l] = skapT[l];
    for (int l = 0; l < NM; ++l) {
      int lp = l + 1, level = l + 1;
      real sigmah = sh[l];
      real zfac = zkonst2 * sigmah * sigmah * vrd[l];
      real dsl = ds[l], dsp = ds[lp];
      real zrthl = (dsp + dsl) / (zte[l] * dsp + zte[lp] * dsl);
      if (level >= ktop && level < ilift) zkdiff[l] = zfac * zrthl * zrthl;
      if (level + 1 == ktop) {
        real zzqs = sat_capped(K, zte[l], dp * sg[l]);
        zzqs = zzqs * (1.0 / (1.0 - K.MOIST * zzqs));
        real zzqsp = sat_capped(K, zte[lp], dp * sg[lp]);
        zzqsp = zzqsp * (1.0 / (1.0 - K.MOIST * zzqsp));
        real zrh = zqe[l] / zzqs, zrhp = zqe[lp] / zzqsp;
        real zzf = std::fabs((zrh - 0.8) / 0.2 * (zrhp - zrh));
        zkdiff[l] = zfac * zrthl * zrthl * zzf;
      }
    }
    real zqn[MAXL], ztn[MAXL];
    for (int l = 0; l < NL; ++l) {
      zqn[l] = zqe[l];
      ztn[l] = zte[l];
    }
    diffuse(NL, ds, zqn, zkdiff);
    for (int l = 0; l < NM; ++l) zkdiff[l] = zkdiff[l] * skaph[l];
    diffuse_potential(NL, ds, ztn, zkdiff, skap);
    for (int l = 0; l < NL; ++l) {
      int at = l * NH + h;
      DTDT[at] = DTDT[at] + (ztn[l] - zte[l]) / K.DELTSEC2;
      DQDT[at] = DQDT[at] + (zqn[l] - zqe[l]) / K.DELTSEC2;
    }
  }
}

// physics/precipitation/wgsl/mkdca.wgsl:1-97 and mkdca-limit.wgsl:1-22.
void mkdca(Model& m) {
  const Consts& K = m.k;
  const int NH = m.NHOR, NL = m.NLEV, NM = m.NLEM;
  const real *skapT = m.TB("vdiff_skap"), *dsT = m.TB("dsigma");
  real *DT = m.F("dt"), *DTDT = m.F("dtdt"), *DQ = m.F("dq"), *DQDT = m.F("dqdt"),
         *DCA_DTDT = m.F("dca_dtdt"), *DCA_DQDT = m.F("dca_dqdt"), *LIM = m.F("dca_limited");
  real skip = 0;
  for (int h = 0; h < NH; ++h) {
    real zt[MAXL], zth[MAXL], zq[MAXL], zqn[MAXL], skap[MAXL], ds[MAXL];
    bool mixed[MAXL] = {false};
    for (int l = 0; l < NL; ++l) {
      int at = l * NH + h;
      skap[l] = skapT[l];
      ds[l] = dsT[l];
      zt[l] = DT[at] + DTDT[at] * K.DELTSEC2;
      zth[l] = zt[l] / skap[l];
      zq[l] = DQ[at] + DQDT[at] * K.DELTSEC2;
      zqn[l] = zq[l];
    }
    real limited = 0;
    int passes = 0;
    for (;;) {
      bool unstable = false;
      int ibase = 0, itop = NL;
      real ztht = 0, zqt = 0, zsum1 = 0, zsum2 = 0, zsumq1 = 0, zsumq2 = 0;
      for (int l = 0; l < NM; ++l) {
        int lp = l + 1;
        if (zth[l] < zth[lp]) {
          ibase = l + 2;
          itop = l;
          zsum1 = skap[lp] * ds[lp] + skap[l] * ds[l];
          zsum2 = skap[lp] * ds[lp] * zth[lp] + skap[l] * ds[l] * zth[l];
          zsumq1 = ds[lp] + ds[l];
          zsumq2 = ds[lp] * zqn[lp] + ds[l] * zqn[l];
          ztht = zsum2 / zsum1;
          zqt = zsumq2 / zsumq1;
          unstable = true;
        }
      }
      if (!unstable) break;
      for (int level = NM - 1; level >= 1; --level) {
        int l = level - 1;
        if (itop == level && zth[l] < ztht) {
          itop = level - 1;
          zsum1 = zsum1 + skap[l] * ds[l];
          zsum2 = zsum2 + skap[l] * ds[l] * zth[l];
          zsumq1 = zsumq1 + ds[l];
          zsumq2 = zsumq2 + ds[l] * zqn[l];
          ztht = zsum2 / zsum1;
          zqt = zsumq2 / zsumq1;
        }
      }
      for (int l = 0; l < NL; ++l) {
        int level = l + 1;
        if (level > itop && level <= ibase) {
          zth[l] = ztht;
          zqn[l] = zqt;
          mixed[l] = true;
        }
      }
      passes = passes + 1;
      if (passes > 2 * NL) {
        limited = 1.0;
        break;
      }
    }
    for (int l = 0; l < NL; ++l) {
      int at = l * NH + h;
      DCA_DTDT[at] = mixed[l] ? (zth[l] * skap[l] - zt[l]) / K.DELTSEC2 : 0.0;
      DCA_DQDT[at] = (zqn[l] - zq[l]) / K.DELTSEC2;
    }
    LIM[h] = limited;
    skip = std::max(skip, limited);
  }
  m.F("dca_skip")[0] = skip;
}

// physics/precipitation/wgsl/column.wgsl + mklsp.wgsl + mkrain.wgsl + mkclouds.wgsl.
void rain_column(Model& m) {
  const Consts& K = m.k;
  const int NH = m.NHOR, NL = m.NLEV;
  const real *ds = m.TB("dsigma"), *sg = m.TB("sigma"), *rcrit = m.TB("rcrit"), *lnsig = m.TB("rad_lnsig");
  real *DTDT = m.F("dtdt"), *DQDT = m.F("dqdt"), *CA_T = m.F("dca_dtdt"), *CA_Q = m.F("dca_dqdt"),
         *DP = m.F("dp"), *DPRSLL = m.F("dprsll"), *DPRLL = m.F("dprll"), *DQ = m.F("dq"), *DT = m.F("dt"),
         *DPRCL = m.F("dprcl"), *DPRSCL = m.F("dprscl"), *DPRC = m.F("dprc"), *DPRL = m.F("dprl"),
         *DPRS = m.F("dprs"), *ICCTOT = m.F("icctot"), *ICCLEV = m.F("icclev"), *DW = m.F("dw"),
         *DQVI = m.F("dqvi"), *DQL = m.F("dql"), *DCC = m.F("dcc");
  const real skip = m.F("dca_skip")[0];
  for (int h = 0; h < NH; ++h) {
    if (skip == 0.0)
      for (int l = 0; l < NL; ++l) {
        int at = l * NH + h;
        DTDT[at] = DTDT[at] + CA_T[at];
        DQDT[at] = DQDT[at] + CA_Q[at];
      }
    // mklsp
    real dp = DP[h];
    for (int l = 0; l < NL; ++l) {
      int at = l * NH + h;
      DPRSLL[at] = 0;
      real dprll = 0, dq = DQ[at];
      real zq = dq + DQDT[at] * K.DELTSEC2;
      real zt = DT[at] + DTDT[at] * K.DELTSEC2;
      real zlcpe = K.ALV / (K.ACPD * (1.0 + K.ADV * dq));
      real p = dp * sg[l];
      real zqsat = sat_capped(K, zt, p);
      real zcor = 1.0 / (1.0 - K.MOIST * zqsat);
      zqsat = zqsat * zcor;
      if (zqsat < 0.0) zqsat = 0.0;
      if (zq > zqsat) {
        real zdqdt = (zqsat - zq) / (1.0 + zlcpe * K.RA2 * (K.TMELT - K.RA4) * zqsat * zcor / ((zt - K.RA4) * (zt - K.RA4)));
        real ztn = zt - zdqdt * zlcpe;
        real zqn = zq + zdqdt;
        zqsat = sat_capped(K, ztn, p);
        zcor = 1.0 / (1.0 - K.MOIST * zqsat);
        zqsat = zqsat * zcor;
        zdqdt = (zqsat - zqn) / (1.0 + zlcpe * K.RA2 * (K.TMELT - K.RA4) * zqsat * zcor / ((ztn - K.RA4) * (ztn - K.RA4)));
        ztn = ztn - zdqdt * zlcpe;
        zqn = zqn + zdqdt;
        real dqdt = (zqn - zq) / K.DELTSEC2, dtdt = (ztn - zt) / K.DELTSEC2;
        DQDT[at] = DQDT[at] + dqdt;
        DTDT[at] = DTDT[at] + dtdt;
        dprll = -std::min(dqdt, 0.0) * ds[l];
      }
      DPRLL[at] = dprll;
    }
    // mkrain
    real zprc = 0, zprl = 0, zprsc = 0, zprsl = 0;
    for (int l = 0; l < NL; ++l) {
      int at = l * NH + h;
      real dsl = ds[l], dq = DQ[at];
      real zdtdt = 0, zdqdtl = 0, zdqdts = 0;
      zprc = zprc + DPRCL[at] - DPRSCL[at];
      zprl = zprl + DPRLL[at] - DPRSLL[at];
      zprsc = zprsc + DPRSCL[at];
      zprsl = zprsl + DPRSLL[at];
      int surface = l == NL - 1 ? 2 : 1;
      for (int below = 0; below < surface; ++below) {
        real temperature = DT[(l + below) * NH + h];
        real zlcp = (K.ALS - K.ALV) / (K.ACPD * (1.0 + K.ADV * dq));
        if (zprsc + zprsl > 0.0 && temperature > K.TMELT) {
          zdtdt = -(zprsc + zprsl) / dsl * zlcp + zdtdt;
          zprc = zprsc + zprc;
          zprl = zprsl + zprl;
          zprsc = 0;
          zprsl = 0;
        } else if (zprc + zprl > 0.0 && temperature <= K.TMELT) {
          zdtdt = (zprc + zprl) / dsl * zlcp + zdtdt;
          zprsc = zprc + zprsc;
          zprsl = zprl + zprsl;
          zprc = 0;
          zprl = 0;
        }
      }
      real zq = dq + DQDT[at] * K.DELTSEC2;
      real zt = DT[at] + DTDT[at] * K.DELTSEC2;
      real zqsat = sat_capped(K, zt, dp * sg[l]);
      real zcor = 1.0 / (1.0 - K.MOIST * zqsat);
      zqsat = zqsat * zcor;
      if (zqsat < 0.0) zqsat = 0.0;
      if (zq < zqsat) {
        real deficit = zqsat - zq;
        real water = K.ALV / (K.ACPD * (1.0 + K.ADV * dq));
        real ice = K.ALS / (K.ACPD * (1.0 + K.ADV * dq));
        auto evap = [&](real& flux, real zlcpe) {
          real zd = std::min(K.GAMMA * deficit * dsl / K.DELTSEC2 /
                                   (1.0 + zlcpe * K.RA2 * (K.TMELT - K.RA4) * zqsat * zcor / ((zt - K.RA4) * (zt - K.RA4))),
                               flux);
          flux = flux - zd;
          return zd / dsl;
        };
        if (zprl > 0.0) {
          real e = evap(zprl, water);
          zdtdt = zdtdt - e * water;
          zdqdtl = zdqdtl + e;
        }
        if (zprc > 0.0) {
          real e = evap(zprc, water);
          zdtdt = zdtdt - e * water;
          zdqdtl = zdqdtl + e;
        }
        if (zprsl > 0.0) {
          real e = evap(zprsl, ice);
          zdtdt = zdtdt - e * ice;
          zdqdts = zdqdts + e;
        }
        if (zprsc > 0.0) {
          real e = evap(zprsc, ice);
          zdtdt = zdtdt - e * ice;
          zdqdts = zdqdts + e;
        }
      }
      DQDT[at] = DQDT[at] + zdqdtl + zdqdts;
      DTDT[at] = DTDT[at] + zdtdt;
    }
    DPRC[h] = (zprc + zprsc) * dp / K.GA / 1000.0;
    DPRL[h] = (zprl + zprsl) * dp / K.GA / 1000.0;
    DPRS[h] = (zprsc + zprsl) * dp / K.GA / 1000.0;
    // mkclouds
    const real ZCLMAX = 1.0, ZCCA = 0.245, ZCCB = 0.125, ZCCMAX = 0.8, ZCCMIN = 0.05;
    real zcctot = ZCCMIN, zccconv = ZCCMIN;
    real dprc = DPRC[h];
    if (dprc > 0.0) {
      zcctot = ZCCA + ZCCB * std::log(dprc * K.ZRFAC);
      zcctot = std::min(ZCCMAX, std::max(ZCCMIN, zcctot));
      real levels = ICCTOT[h];
      zccconv = levels == 0.0 ? 1.0 : 1.0 - fpow(1.0 - zcctot, 1.0 / levels);
    }
    real cover[MAXL];
    for (int l = 0; l < NL; ++l) {
      int at = l * NH + h;
      real zt = DT[at] + DTDT[at] * K.DELTSEC2;
      real zq = DQ[at] + DQDT[at] * K.DELTSEC2;
      real zqsat = sat_divided(K, zt, dp * sg[l]);
      real zrh = zq / zqsat;
      real icclev = ICCLEV[at];
      real dcc = icclev > 0.0 ? zccconv : 0.0;
      if (icclev == 2.0 && zcctot >= 0.3) dcc = std::min(dcc + 2.0 * (zcctot - 0.3), ZCLMAX);
      zrh = zrh * (1.0 - dcc);
      real zrcrit = rcrit[l];
      real zwfac = 1.0;
      if (sg[l] > 0.8 && K.CLWFAC > 0.0) {
        real dw = DW[at];
        zwfac = K.CLWFAC * std::max(0.0, K.CLWCRIT1 - dw);
        if (K.CLWCRIT2 > dw) zwfac = 1.0;
      }
      real excess = std::max(0.0, (zrh - zrcrit) / (1.0 - zrcrit));
      cover[l] = std::min(dcc + zwfac * (excess * excess), ZCLMAX);
    }
    real zzf[MAXL];
    real dqvi = 0, zzh = 0;
    for (int l = NL - 1; l >= 1; --l) {
      dqvi = DQ[l * NH + h] * ds[l] + dqvi;
      real zdh = -DT[l * NH + h] * K.GASCON / K.GA * lnsig[l];
      zzf[l] = zzh + zdh * 0.5;
      zzh = zzh + zdh;
    }
    dqvi = DQ[h] * ds[0] + dqvi;
    zzf[0] = zzh - DT[h] * K.GASCON / K.GA * lnsig[0];
    dqvi = dqvi * dp / K.GA;
    DQVI[h] = dqvi;
    zzh = 700.0 * std::log(1.0 + dqvi);
    real clear = 1.0;
    for (int l = 0; l < NL; ++l) {
      int at = l * NH + h;
      real dql = 0;
      if (zzh > 0.0 && cover[l] > 0.0) {
        dql = 0.00021 * std::exp(-zzf[l] / zzh) * K.GASCON * DT[at] / (sg[l] * dp);
        dql = std::max(dql, 1.0e-9);
      }
      DQL[at] = dql;
      DCC[at] = cover[l];
      clear = clear * (1.0 - cover[l]);
    }
    DQL[NL * NH + h] = 0;
    DCC[NL * NH + h] = 1.0 - clear;
  }
}

// ----------------------------------------------------------------- surface
// physics/land/wgsl/soil.wgsl:1-185 (soilstep: tands, mktsoil, wandr).
void soil(Model& m) {
  const Consts& K = m.k;
  const int NH = m.NHOR, NLS = 5;
  const real* dsoilz = m.TB("dsoilz");
  real *DLS = m.F("dls"), *DSNOWZ = m.F("dsnowz"), *DSNOWT = m.F("dsnowt"), *DGLAC = m.F("dglac"),
         *DSHFL = m.F("dshfl"), *DLHFL = m.F("dlhfl"), *DFLUX = m.F("dflux"), *DEVAP = m.F("devap"),
         *DPRS = m.F("dprs"), *DPRL = m.F("dprl"), *DPRC = m.F("dprc"), *LAND_DTSM = m.F("land_dtsm"),
         *DSOILT = m.F("dsoilt"), *LAND_DTS = m.F("land_dts"), *DSNDCH = m.F("dsndch"), *DWATER = m.F("dwater"),
         *DSMELT = m.F("dsmelt"), *DWATC = m.F("dwatc"), *DWMAX = m.F("dwmax"), *DRUNOFF = m.F("drunoff");
  struct Layer {
    real ctop, soilz1, diff1, cap1;
  };
  auto snow_layer = [&](real snowz, real cap0, real diff0, real soilz0) {
    real zsntop = std::min(snowz * 1000.0 / K.RHOSNOW, K.DZTOP);
    real ctop = cap0 * K.SNOWCAP * K.DZTOP / (cap0 * zsntop + K.SNOWCAP * (K.DZTOP - zsntop));
    real zsnowz = std::min(snowz * 1000.0 / K.RHOSNOW, 1.0) - zsntop;
    real soilz1 = soilz0 + zsnowz;
    real diff1 = diff0 * K.SNOWDIFF * soilz1 / (K.SNOWDIFF * soilz0 + diff0 * zsnowz);
    real cap1 = cap0 * K.SNOWCAP * soilz1 / (cap0 * zsnowz + K.SNOWCAP * soilz0);
    return Layer{ctop, soilz1, diff1, cap1};
  };
  auto surface_temperature = [&](const Layer& ly, real dtsm, real flux, real soil1) {
    real conduction = 2.0 * ly.diff1;
    return (ly.ctop * K.DZTOP * dtsm / K.DELTSEC + flux + conduction * soil1 / ly.soilz1) /
           (ly.ctop * K.DZTOP / K.DELTSEC + conduction / ly.soilz1);
  };
  for (int h = 0; h < NH; ++h) {
    real dls = DLS[h];
    bool land = dls > 0.0;
    real snowStart = DSNOWZ[h];
    real dwater = 0, dsmelt = 0;
    if (snowStart == 0.0) DSNOWT[h] = K.TMELT;
    if (land) {
      real glac = DGLAC[h];
      real soilz[NLS], cap[NLS], diff[NLS];
      for (int l = 0; l < NLS; ++l) {
        cap[l] = K.SICECAP * glac + K.SOILCAP * (1.0 - glac);
        diff[l] = K.SICEDIFF * glac + K.SOILDIFF * (1.0 - glac);
        soilz[l] = dsoilz[l];
      }
      real zhfla = DSHFL[h] + DLHFL[h] + DFLUX[m.NLEV * NH + h];
      real devap = DEVAP[h];
      real zdsnowz = 0;
      if (DPRS[h] > 0.0) zdsnowz = DPRS[h];
      if (snowStart > 0.0) zdsnowz = zdsnowz + devap;
      real zsnowz = std::max(0.0, snowStart + zdsnowz * K.DELTSEC);
      zdsnowz = (zsnowz - snowStart) / K.DELTSEC;
      dwater = devap + DPRL[h] + DPRC[h] - zdsnowz;
      real dsnowz = zsnowz;
      real dtsm = LAND_DTSM[h], soil1 = DSOILT[h];
      Layer layer = snow_layer(dsnowz, cap[0], diff[0], soilz[0]);
      real dts = surface_temperature(layer, dtsm, zhfla, soil1);
      real zhfls = 2.0 * layer.diff1 / layer.soilz1 * (dts - soil1);
      real zhflm = 0;
      if (dsnowz > 0.0 && dts > K.TMELT) {
        dts = K.TMELT;
        zhflm = std::max(0.0, zhfla - layer.ctop * K.DZTOP * (dts - dtsm) / K.DELTSEC +
                                  2.0 * layer.diff1 * (soil1 - dts) / layer.soilz1);
        zsnowz = std::max(0.0, dsnowz - zhflm * K.DELTSEC / ((K.ALS - K.ALV) * 1000.0));
        zdsnowz = (zsnowz - dsnowz) / K.DELTSEC;
        zhflm = -zdsnowz * 1000.0 * (K.ALS - K.ALV);
        dsnowz = zsnowz;
        dsmelt = -zdsnowz;
        zhfls = 2.0 * layer.diff1 / layer.soilz1 * (dts - soil1);
        dwater = dwater - zdsnowz;
        layer = snow_layer(dsnowz, cap[0], diff[0], soilz[0]);
      }
      if (dsnowz == 0.0 && zhflm > 0.0) {
        dts = surface_temperature(layer, dtsm, zhfla - zhflm, soil1);
        zhfls = 2.0 * layer.diff1 / layer.soilz1 * (dts - soil1);
      }
      soilz[0] = layer.soilz1;
      cap[0] = layer.cap1;
      diff[0] = layer.diff1;
      // mktsoil
      real zdiff[NLS], zcap[NLS], zebs[NLS], ztn[NLS];
      int n = NLS - 1;
      zdiff[n - 1] = 2.0 * diff[n] * diff[n - 1] / (diff[n] * soilz[n - 1] + diff[n - 1] * soilz[n]);
      zcap[n] = cap[n] * soilz[n] / K.DELTSEC;
      zebs[n] = 1.0 / (zcap[n] + zdiff[n - 1]);
      ztn[n] = zcap[n] * DSOILT[n * NH + h] * zebs[n];
      for (int l = n - 1; l >= 1; --l) {
        zdiff[l - 1] = 2.0 * diff[l] * diff[l - 1] / (diff[l] * soilz[l - 1] + diff[l - 1] * soilz[l]);
        zcap[l] = cap[l] * soilz[l] / K.DELTSEC;
        zebs[l] = 1.0 / (zcap[l] + zdiff[l - 1] + zdiff[l] * (1.0 - zdiff[l] * zebs[l + 1]));
        ztn[l] = zebs[l] * (zcap[l] * DSOILT[l * NH + h] + zdiff[l] * ztn[l + 1]);
      }
      zcap[0] = cap[0] * soilz[0] / K.DELTSEC;
      zebs[0] = 1.0 / (zcap[0] + zdiff[0] * (1.0 - zdiff[0] * zebs[1]));
      ztn[0] = zebs[0] * (zcap[0] * DSOILT[h] + zdiff[0] * ztn[1] + zhfls);
      for (int l = 1; l < NLS; ++l) ztn[l] = ztn[l] + zebs[l] * zdiff[l - 1] * ztn[l - 1];
      bool glacier = DGLAC[h] > 0.5;
      for (int l = 0; l < NLS; ++l) DSOILT[l * NH + h] = glacier ? std::min(ztn[l], K.TMELT) : ztn[l];
      if (dsnowz > 0.0) DSNOWT[h] = dts;
      if (K.DSMAX > 0.0 && dsnowz > K.DSMAX) {
        zdsnowz = (K.DSMAX - dsnowz) / K.DELTSEC;
        dsnowz = K.DSMAX;
        dwater = dwater - zdsnowz;
        dts = dts + zdsnowz * 1000.0 * (K.ALS - K.ALV) * K.DELTSEC / layer.ctop / K.DZTOP;
        dsmelt = dsmelt - zdsnowz;
      }
      DSNOWZ[h] = dsnowz;
      LAND_DTS[h] = dts;
      DSNDCH[h] = dsnowz - snowStart;
    } else {
      DSNDCH[h] = snowStart;
    }
    DWATER[h] = dwater;
    DSMELT[h] = dsmelt;
    real drunoff = 0;
    if (land) {
      real dwatc = DWATC[h] + K.DELTSEC * dwater;
      real dwmax = DWMAX[h];
      drunoff = std::max(0.0, dwatc - dwmax) / K.DELTSEC;
      DWATC[h] = std::max(std::min(dwmax, dwatc), 0.0);
    }
    DRUNOFF[h] = drunoff;
  }
}

// physics/land/wgsl/mkradv.wgsl:1-59 (river routing; reads only driver).
void mkradv(Model& m) {
  const int NH = m.NHOR, NLON = m.NLON, NLAT = m.NLAT;
  real *DRIVER = m.F("driver"), *DAREA = m.F("darea"), *DLS = m.F("dls"), *DUROFF = m.F("duroff"),
         *DVROFF = m.F("dvroff"), *DRUNOFF = m.F("drunoff");
  std::vector<real> out(NH);
  auto river = [&](int h) { return DRIVER[h] * DAREA[h] * DLS[h]; };
  auto eastward = [&](int row, int lon, real& o, real& in) {
    int h = row + lon, nx = row + (lon + 1) % NLON;
    real u = DUROFF[h];
    real water = u > 0.0 ? river(h) : river(nx);
    o = u * water / DAREA[h];
    in = u * water / DAREA[nx];
  };
  for (int h = 0; h < NH; ++h) {
    int lat = h / NLON, lon = h % NLON, row = lat * NLON;
    real runoff = DRUNOFF[h], o, in;
    if (lon == 0) {
      eastward(row, 0, o, in);
      runoff = runoff - o;
      eastward(row, NLON - 1, o, in);
      runoff = runoff + in;
    } else {
      eastward(row, lon - 1, o, in);
      runoff = runoff + in;
      eastward(row, lon, o, in);
      runoff = runoff - o;
    }
    real area = DAREA[h], v = DVROFF[h];
    real below = lat + 1 < NLAT ? river(h + NLON) : 0.0;
    if (v < 0.0)
      runoff = runoff + v * river(h) / area;
    else
      runoff = runoff + v * below / area;
    real fromAbove = 0;
    if (lat > 0) {
      int above = h - NLON;
      real va = DVROFF[above];
      fromAbove = va < 0.0 ? -va * river(above) : -va * river(h);
    }
    out[h] = runoff + fromAbove / area;
  }
  for (int h = 0; h < NH; ++h) DRUNOFF[h] = out[h];
}

// physics/land/wgsl/surface.wgsl:1-142 with vegetation/wgsl/vegstep.wgsl:1-99 and
// glacier/wgsl/glacierstep.wgsl:1-25.
void land_surface(Model& m) {
  const Consts& K = m.k;
  const int NH = m.NHOR, NL = m.NLEV;
  real *DLS = m.F("dls"), *DRIVER = m.F("driver"), *DRUNOFF = m.F("drunoff"), *LAND_DTS = m.F("land_dts"),
         *SS = m.F("surface_step"), *DALBCL = m.F("dalbcl"), *DALBCL1 = m.F("dalbcl1"), *DALBCL2 = m.F("dalbcl2"),
         *DWATER = m.F("dwater"), *DALBCLIM = m.F("dalbclim"), *DALBCLIM1 = m.F("dalbclim1"),
         *DALBCLIM2 = m.F("dalbclim2"), *LAND_DTSM = m.F("land_dtsm"), *DP = m.F("dp"), *LAND_DQS = m.F("land_dqs"),
         *DSNOWZ = m.F("dsnowz"), *DSNOW = m.F("dsnow"), *DFOREST = m.F("dforest"), *DALB = m.F("dalb"),
         *DSALB = m.F("dsalb"), *DRHS = m.F("drhs"), *DWMAX = m.F("dwmax"), *DWATC = m.F("dwatc"),
         *DTSOIL = m.F("dtsoil"), *DTD2 = m.F("dtd2"), *DTD3 = m.F("dtd3"), *DTD4 = m.F("dtd4"), *DTD5 = m.F("dtd5"),
         *DSOILT = m.F("dsoilt"), *DT = m.F("dt"), *DQ = m.F("dq"), *DGLAC = m.F("dglac"), *DPERSIST = m.F("dpersist");
  real *CO2 = m.F("co2"), *DCVEG = m.F("dcveg"), *DCSOIL = m.F("dcsoil"), *DAGG = m.F("dagg"), *DFD = m.F("dfd"),
         *DEVAP = m.F("devap"), *DGROW = m.F("dgrow"), *DNPP = m.F("dnpp"), *DVSOIL = m.F("dvsoil"),
         *DLAI = m.F("dlai"), *DMR = m.F("dmr"), *DSC = m.F("dsc"), *DZ0CLIMO = m.F("dz0climo"), *DZ0 = m.F("dz0");
  auto clim = [&](const real* f, int h) {
    real w = SS[5];
    return (1.0 - w) * f[(int)SS[3] * NH + h] + w * f[(int)SS[4] * NH + h];
  };
  auto snow_albedo = [&](real forest, real mxf, real mxb, real mnf, real mnb, real ts) {
    real zmax = forest * mxf + (1.0 - forest) * mxb;
    real zmin = forest * mnf + (1.0 - forest) * mnb;
    real zd = (zmax - zmin) * (ts - 263.16) / (K.TMELT - 263.16);
    return std::max(zmin, std::min(zmax, zmax - zd));
  };
  auto glacier_albedo = [&](real mx, real mn, real ts) {
    return std::max(mn, std::min(mx, mx - (mx - mn) * (ts - 263.16) / (K.TMELT - 263.16)));
  };
  for (int h = 0; h < NH; ++h) {
    real dls = DLS[h];
    if (dls > 0.0) DRIVER[h] = DRIVER[h] + DRUNOFF[h] * K.DELTSEC;
    real dts = LAND_DTS[h];
    real albclim = clim(DALBCL, h), albclim1 = clim(DALBCL1, h), albclim2 = clim(DALBCL2, h);
    if (K.NWETSOIL != 0 && dls > 0.5) {
      if (dts > 273.15) {
        real bf = DWATER[h] / K.WSMAX;
        real al = 1.0 / 5.2 * fpow(fpow(std::max(bf, 1.0e-3), (1.0 - 4.0) / 4.0) - 1.0, 1.0 / 4.0);
        real dry = std::exp(-powi(bf * 25.0, 6));
        real wet = std::exp(-powi((1.0 - bf) * 30.0, 9));
        albclim = K.ALBLANDMAX * dry + al * (1.0 - dry - wet) + K.DOCEANALB1 * wet;
        albclim1 = albclim;
        albclim2 = K.ALBLANDMAX * dry + al * (1.0 - dry - wet) + K.DOCEANALB2 * wet;
      } else {
        albclim = K.ALBLAND;
        albclim1 = K.DGROUNDALB1;
        albclim2 = K.DGROUNDALB2;
      }
    }
    DALBCLIM[h] = albclim;
    DALBCLIM1[h] = albclim1;
    DALBCLIM2[h] = albclim2;
    if (dls > 0.0) {
      LAND_DTSM[h] = dts;
      real dqs = K.RDBRV * K.RA1 * std::exp(K.RA2 * (dts - K.TMELT) / (dts - K.RA4)) / DP[h];
      dqs = dqs / (1.0 - (1.0 / K.RDBRV - 1.0) * dqs);
      LAND_DQS[h] = dqs;
      real dsnow = DSNOWZ[h];
      DSNOW[h] = dsnow;
      if (dsnow > 0.0) {
        real forest = DFOREST[h];
        real s0 = snow_albedo(forest, K.ALBSMAXF, K.ALBSMAX, K.ALBSMINF, K.ALBSMIN, dts);
        real s1 = snow_albedo(forest, K.ALBSMAXF1, K.ALBSMAX1, K.ALBSMINF1, K.ALBSMIN1, dts);
        real s2 = snow_albedo(forest, K.ALBSMAXF2, K.ALBSMAX2, K.ALBSMINF2, K.ALBSMIN2, dts);
        DALB[h] = albclim + (s0 - albclim) * dsnow / (dsnow + 0.01);
        DSALB[h] = albclim1 + (s1 - albclim1) * dsnow / (dsnow + 0.01);
        DSALB[NH + h] = albclim2 + (s2 - albclim2) * dsnow / (dsnow + 0.01);
        DRHS[h] = 1.0;
      } else {
        DALB[h] = albclim;
        DSALB[h] = albclim1;
        DSALB[NH + h] = albclim2;
        real dwmax = DWMAX[h];
        if (dwmax > 0.0) DRHS[h] = std::min(1.0, DWATC[h] / (K.DRHSFULL * dwmax));
      }
      DTSOIL[h] = DSOILT[h];
      DTD2[h] = DSOILT[NH + h];
      DTD3[h] = DSOILT[2 * NH + h];
      DTD4[h] = DSOILT[3 * NH + h];
      DTD5[h] = DSOILT[4 * NH + h];
      DT[NL * NH + h] = dts;
      DQ[NL * NH + h] = dqs;
    }
    if (K.NVEG > 0 && DLS[h] > 0.0 && DGLAC[h] < 0.90) {
      // vegstep
      real co2 = CO2[0];
      real zbeta = 0;
      if (!(co2 < 1.0e-8))
        zbeta = std::max(0.0, 1.0 + K.CO2_SENS * std::log((co2 - K.CO2_COMP) / (K.CO2_REF - K.CO2_COMP)));
      real ts = DT[NL * NH + h], dp = DP[h], dwatc = DWATC[h], dsnow = DSNOW[h];
      real zwmax = DWMAX[h];
      real zglacfree = 1.0 - DGLAC[h];
      real zsvp = K.RA1 * std::exp(K.RA2 * (ts - K.TMELT) / (ts - K.RA4));
      real zvpd = std::max(0.01, zsvp - dp * DQ[(NL - 1) * NH + h] / 0.622);
      real dcveg = DCVEG[h], dcsoil = DCSOIL[h];
      real zlaim = K.ZLAIMIN + 0.63661977236758 * K.ZLAIMAX * std::atan(K.CVEG_L * 2.0 * DAGG[h] * dcveg);
      real zvegm = 1.0 - std::exp(-K.CVEG_K * zlaim);
      real zveg = 0;
      if (zwmax > 0.0) zveg = std::min(std::min(1.0, zvegm), std::max(0.0, dwatc / (zwmax * K.VWS_CRIT)));
      real zft = std::min(1.0, std::max(0.0, (ts - K.TMELT) / K.CT_CRIT));
      real zgppl = K.RLUE * zbeta * zft * zveg * DFD[NL * NH + h];
      real zgppw = 0;
      if (!(co2 < 1.0e-8)) zgppw = K.CO2CONV * dp * zveg * (-DEVAP[h]) / zvpd * (0.3 * co2);
      zgppw = std::min(1.0, std::max(0.0, zgppw));
      real zgpp = std::min(zgppl, zgppw);
      real znpp = DGROW[h] * 0.5 * zgpp * zglacfree;
      DNPP[h] = znpp;
      real zlitter = dcveg / K.TAU_VEG;
      real zres = fpow(K.Q10, (ts - K.TMELT - 10.0) / 10.0) * dcsoil / K.TAU_SOIL;
      dcveg = dcveg + (znpp - zlitter) * K.DELTSEC * K.NCVEG;
      dcsoil = dcsoil + (zlitter - zres) * K.DELTSEC * K.NCVEG;
      real zforest = std::min(1.0, std::max(0.0, (std::atan(dcveg - K.CVEG_A) - K.CVEG_E) / (K.CVEG_C - K.CVEG_E)));
      real dvsoil = std::min(1.0, std::max(0.0, (std::atan(dcveg - K.CVEG_F) - K.CVEG_G) / (K.CVEG_C - K.CVEG_G)));
      DCVEG[h] = dcveg;
      DCSOIL[h] = dcsoil;
      DVSOIL[h] = dvsoil;
      DLAI[h] = -std::log(1.0 - zveg) / K.CVEG_K;
      real zvz0 = DMR[h] * zforest + K.VZ0_MIN * (1.0 - zforest);
      real zvalb = K.VALB_MIN * zveg + K.VALB_MAX * (1.0 - zveg);
      zwmax = K.VWMAX_MAX * dvsoil + K.VWMAX_MIN * (1.0 - dvsoil);
      real zvrhs = DSC[h] * std::min(1.0, std::max(0.0, dwatc / (zwmax * K.VWS_CRIT)));
      if (dsnow > 0.0) {
        real zalbsn = (K.ALBSMAX - K.ALBSMIN) * (ts - 263.16) / (K.TMELT - 263.16);
        zalbsn = std::max(K.ALBSMIN, std::min(K.ALBSMAX, K.ALBSMAX - zalbsn));
        zvalb = zvalb + (zalbsn - zvalb) * dsnow / (dsnow + 0.01);
        zvalb = K.VSALB_MIN * zforest + zvalb * (1.0 - zforest);
        zvrhs = 1.0;
      }
      if (K.NVEG == 2) {
        real z0c = DZ0CLIMO[h];
        DZ0[h] = std::sqrt(zvz0 * zvz0 + z0c * z0c);
        DWMAX[h] = zwmax;
        DRHS[h] = zvrhs;
        DALB[h] = zvalb;
        DFOREST[h] = zforest;
      }
    }
    if (DGLAC[h] > 0.5 && dls > 0.0) {
      DALB[h] = glacier_albedo(K.ALBGMAX, K.ALBGMIN, dts);
      DSALB[h] = glacier_albedo(K.ALBGMAX1, K.ALBGMIN1, dts);
      DSALB[NH + h] = glacier_albedo(K.ALBGMAX2, K.ALBGMIN2, dts);
      DRHS[h] = 1.0;
    }
    if (K.NGLACIER != 0) {
      bool lnd = DLS[h] > 0.5;
      if (lnd && DSNOWZ[h] < K.GLACELIM) DPERSIST[h] = 0.0;
      if (lnd && DSNOWZ[h] < 0.1) DGLAC[h] = 0.0;
      if (SS[6] > 0.5) {
        if (DPERSIST[h] > 0.5) DGLAC[h] = 1.0;
        DPERSIST[h] = DLS[h] >= 0.5 ? 1.0 : 0.0;
      }
    }
  }
}

// physics/sea-ice/wgsl/ice.wgsl:1-225 and the getiflx sums (reduction/wgsl/sum.wgsl).
void sea_ice(Model& m) {
  const Consts& K = m.k;
  const int NH = m.NHOR, NL = m.NLEV;
  real *DLS = m.F("dls"), *NACC = m.F("sea_naccua"), *DSHFL = m.F("dshfl"), *DSWFL = m.F("dswfl"),
         *DLWFL = m.F("dlwfl"), *DLHFL = m.F("dlhfl"), *CHEATA = m.F("sea_cheata"), *DPRS = m.F("dprs"),
         *CPRSA = m.F("sea_cprsa"), *SS = m.F("surface_step"), *XCLSSTO = m.F("xclssto"), *XCLSST = m.F("xclsst"),
         *XCLSST2 = m.F("xclsst2"), *XCLICED = m.F("xcliced"), *XCLICEC = m.F("xclicec"), *XCLICED2 = m.F("xcliced2"),
         *XCLICEC2 = m.F("xclicec2"), *XLS = m.F("xls"), *XSST = m.F("xsst"), *XICED = m.F("xiced"),
         *XSNOW = m.F("xsnow"), *XICECC = m.F("xicecc"), *XCFLUX = m.F("xcflux"), *XCFLUXF = m.F("xcfluxf"),
         *SNOWOLD = m.F("ice_snowold"), *XICEC = m.F("xicec"), *XTS = m.F("xts"), *XQMELT = m.F("xqmelt"),
         *XOFLUX = m.F("xoflux"), *ZFLX = m.F("ice_zflx"), *XGW = m.F("xgw"), *P1 = m.F("ice_part1"),
         *P2 = m.F("ice_part2"), *XCFLUXR = m.F("xcfluxr"), *XIMELT = m.F("ximelt"), *XSMELT = m.F("xsmelt"),
         *XSMFLX = m.F("xsmflx"), *XSNDCH = m.F("xsndch"), *SUMS = m.F("ice_sums");
  auto clim = [&](const real* f, int h, int off) {
    real w = SS[off + 2];
    return (1.0 - w) * f[(int)SS[off] * NH + h] + w * f[(int)SS[off + 1] * NH + h];
  };
  for (int h = 0; h < NH; ++h) {
    bool sea = DLS[h] < 0.5;
    real xheat = 0, xprs = 0;
    if (sea) {
      real naccua = NACC[h] + 1.0;
      xheat = (DSHFL[h] + DSWFL[NL * NH + h] + DLWFL[NL * NH + h] + DLHFL[h] + CHEATA[h]) / naccua;
      xprs = (DPRS[h] + CPRSA[h]) / naccua;
    }
    CHEATA[h] = 0;
    CPRSA[h] = 0;
    NACC[h] = 0;
    real zrhoilfdt = K.CRHOI * K.CLFI / K.XDT;
    XCLSSTO[h] = clim(XCLSST, h, 0);
    XCLSST2[h] = clim(XCLSST, h, 3);
    real cliced = std::max(clim(XCLICED, h, 3), 0.0);
    real clicec = std::max(clim(XCLICEC, h, 3), 0.0);
    if (cliced <= 0.0) clicec = 0.0;
    XCLICED2[h] = cliced;
    XCLICEC2[h] = clicec;
    real xls = XLS[h], xsst = XSST[h], xiced = XICED[h], xsnow = XSNOW[h], xicecc = XICECC[h],
           xcflux = XCFLUX[h], xcfluxf = XCFLUXF[h];
    SNOWOLD[h] = xsnow;
    real zicedold = xls < 0.5 ? xiced : 0.0;
    real ximelt = 0, xsmelt = 0, xsmflx = 0, xscflx = 0, xsndch = 0, xcfluxr = 0;
    if (XICEC[h] >= K.CICEMIN) {
      xsnow = xsnow + xprs * K.XDT;
      xprs = 0;
    }
    real xts = XTS[h], xqmelt = 0;
    real ztso = std::min(K.TMELT, xts);
    real zhsnow = 1.0e3 / K.CRHOSN * xsnow;
    if (xiced >= K.XMIND) {
      real zcpdt = K.XMIND * K.CRHOI * K.CPI / K.XDT;
      real zckap = (K.CKAPSN * zhsnow + K.CKAPI * xiced) / (zhsnow + xiced);
      real zkapz = zckap / (xiced + zhsnow);
      if (xiced >= K.XMAXD && K.XMAXD >= 0.0) zkapz = 0.0;
      real zflx = xheat + zkapz * xsst;
      xts = (zcpdt * ztso + zflx) / (zcpdt + zkapz);
      if (xts > K.TMELT) {
        xqmelt = xheat + zkapz * (xsst - K.TMELT) - zcpdt * (K.TMELT - ztso);
        xts = K.TMELT;
      }
    } else {
      xts = xsst;
      if (xiced > 0.0) xqmelt = xheat;
    }
    XTS[h] = xts;
    XQMELT[h] = xqmelt;
    if (xiced < K.XMIND) {
      xcflux = xheat;
      xcfluxf = 0.0;
    } else {
      real zhsnowc = 1.0e3 / K.CRHOSN * xsnow;
      real zckap = (K.CKAPSN * zhsnowc + K.CKAPI * xiced) / (zhsnowc + xiced);
      if (K.XMAXD >= 0.0 && xiced >= K.XMAXD) zckap = 0.0;
      xcflux = zckap * (xts - xsst) / (zhsnowc + xiced);
      xcfluxf = zckap * (K.TFREEZE - xsst) / (zhsnowc + xiced);
    }
    if (XICEC[h] < K.CICEMIN && xprs > 0.0) {
      xcflux = xcflux - xprs * 1000.0 * K.CLFSN;
      xsmelt = xprs + xsmelt;
      xsmflx = xsmflx + xprs * 1000.0 * K.CLFSN;
      xprs = 0;
    }
    real zqmelt = xqmelt;
    if (xiced > 0.0) {
      if (xqmelt > xsnow * 1000.0 * K.CLFSN / K.XDT) {
        xsmelt = xsmelt + xsnow / K.XDT;
        xsmflx = xsmflx + xsnow * 1000.0 * K.CLFSN / K.XDT;
        zqmelt = xqmelt - xsnow * 1000.0 * K.CLFSN / K.XDT;
        xsnow = 0;
      } else if (xqmelt > 0.0 && xsnow > 0.0) {
        xsmelt = xsmelt + xqmelt / K.CLFSN / 1000.0;
        xsnow = xsnow - xqmelt * K.XDT / K.CLFSN / 1000.0;
        xsmflx = xsmflx + xqmelt;
        zqmelt = 0;
      }
      xcflux = xcflux + zqmelt;
    } else {
      xsmelt = xsmelt + xsnow / K.XDT;
      xcflux = xcflux - xsnow * 1000.0 * K.CLFSN / K.XDT;
      xsmflx = xsmflx + xsnow * 1000.0 * K.CLFSN / K.XDT;
      xsnow = 0;
    }
    if (xls < 0.5 && 1.0e3 * xsnow > (K.CRHOS - K.CRHOI) * xiced) {
      real zhice = (1.0e3 * xsnow + K.CRHOI * xiced) / K.CRHOS;
      real zdice = zhice - xiced;
      real zdsnow = -zdice * K.CRHOI / 1.0e3;
      xsnow = xsnow + zdsnow;
      xscflx = zdsnow * 1.0e3 * K.CLFSN / K.XDT;
      xsmelt = xsmelt - zdsnow / K.XDT;
      xsmflx = xsmflx - zdsnow * 1.0e3 * K.CLFSN / K.XDT;
    }
    if (xls < 0.5) xcflux = xcflux + XOFLUX[h];
    if (xsst <= K.TFREEZE || xiced > 0.0) {
      ximelt = xcflux + xscflx - xcfluxf;
      xiced = xiced - ximelt / zrhoilfdt;
      xcflux = xcfluxf;
    }
    if (xiced <= 0.0) {
      xcflux = xcflux - xiced * zrhoilfdt;
      ximelt = ximelt + xiced * zrhoilfdt;
      xiced = 0;
    }
    if (std::fabs(xiced) < 1.0e-9) xiced = 0;
    if (xiced > zicedold) xicecc = std::min(xicecc + (1.0 - xicecc) * (xiced - zicedold) / 0.5, 1.0);
    if (xiced < zicedold) xicecc = std::max(xicecc + xicecc * (xiced - zicedold) / (2.0 * zicedold), 0.0);
    if (xiced <= 0.0) xicecc = 0;
    if (K.XMAXD >= 0.0 && xiced > K.XMAXD) {
      real zcflux = (xiced - K.XMAXD) * zrhoilfdt;
      xiced = K.XMAXD;
      xcfluxr = xcfluxr + zcflux;
      ximelt = ximelt + zcflux;
      xsndch = xsndch + zcflux * 1000.0 / K.CRHOI / zrhoilfdt;
    }
    real zflx = ZFLX[h];
    if (xls < 1.0) zflx = std::max(0.0, K.XMAXD - xiced) * zrhoilfdt;
    ZFLX[h] = zflx;
    real xgw = XGW[h];
    P1[h] = xls < 1.0 ? xcfluxr * xgw : 0.0;
    P2[h] = xls < 1.0 ? zflx * xgw : 0.0;
    XICED[h] = xiced;
    XSNOW[h] = xsnow;
    XICECC[h] = xicecc;
    XICEC[h] = xicecc;
    XCFLUX[h] = xcflux;
    XCFLUXF[h] = xcfluxf;
    XCFLUXR[h] = xcfluxr;
    XIMELT[h] = ximelt;
    XSMELT[h] = xsmelt;
    XSMFLX[h] = xsmflx;
    XSNDCH[h] = xsndch;
  }
  real a = 0, b = 0;
  for (int h = 0; h < NH; ++h) {
    a += P1[h];
    b += P2[h];
  }
  SUMS[0] = a;
  SUMS[1] = b;
}

// physics/sea/wgsl/seastep.wgsl:1-75 with sea-ice/wgsl/finish.wgsl:1-46 and
// ocean/wgsl/oceanstep.wgsl:1-46.
void sea(Model& m) {
  const Consts& K = m.k;
  const int NH = m.NHOR, NL = m.NLEV;
  const bool coupled = K.ICE_COUPLED != 0;
  real *XLS = m.F("xls"), *XCFLUX = m.F("xcflux"), *XCFLUXR = m.F("xcfluxr"), *SUMS = m.F("ice_sums"),
         *ZFLX = m.F("ice_zflx"), *XICED = m.F("xiced"), *XICEC = m.F("xicec"), *XSNOW = m.F("xsnow"),
         *XSMELT = m.F("xsmelt"), *XSMFLX = m.F("xsmflx"), *XOFLUX = m.F("xoflux"), *XOHEAT = m.F("xoheat"),
         *XSNDCH = m.F("xsndch"), *SNOWOLD = m.F("ice_snowold"), *SS = m.F("surface_step"), *YCLSST = m.F("yclsst"),
         *YCLSST2 = m.F("yclsst2"), *YLS = m.F("yls"), *YMLD = m.F("ymld"), *YFLDO = m.F("yfldo"), *YSST = m.F("ysst"),
         *XSST = m.F("xsst"), *XMLD = m.F("xmld"), *NACC = m.F("sea_naccua"), *DLS = m.F("dls"), *XTS = m.F("xts"),
         *SEA_DSST = m.F("sea_dsst"), *SEA_DTS = m.F("sea_dts"), *DMLD = m.F("dmld"), *DICEC = m.F("dicec"),
         *DICED = m.F("diced"), *DSNOW = m.F("dsnow"), *DSMELT = m.F("dsmelt"), *DSNDCH = m.F("dsndch"),
         *CHEATA = m.F("sea_cheata"), *DSHFL = m.F("dshfl"), *DSWFL = m.F("dswfl"), *DLWFL = m.F("dlwfl"),
         *DLHFL = m.F("dlhfl"), *CPRSA = m.F("sea_cprsa"), *DPRS = m.F("dprs"), *DP = m.F("dp"), *DT = m.F("dt"),
         *DQ = m.F("dq"), *SEA_DQS = m.F("sea_dqs"), *DTAUX = m.F("dtaux"), *DTAUY = m.F("dtauy"),
         *DRHS = m.F("drhs"), *DALB = m.F("dalb"), *DSALB = m.F("dsalb"), *DZ0 = m.F("dz0");
  for (int h = 0; h < NH; ++h) {
    if (coupled) {
      // ice_finish
      real xls = XLS[h], xcflux = XCFLUX[h], xcfluxr = XCFLUXR[h], s1 = SUMS[0], s2 = SUMS[1];
      if (s1 > 0.0 && s2 > 0.0 && xls < 1.0) {
        real zflx = ZFLX[h];
        real zfac = s1 / s2;
        if (zfac <= 1.0) zflx = zflx * zfac;
        xcfluxr = xcfluxr - zflx;
        xcflux = xcflux - zflx;
      }
      XCFLUXR[h] = xcfluxr;
      real xiced = XICED[h];
      real xicec = XICEC[h] >= K.THICEC ? 1.0 : 0.0;
      real xsnow = XSNOW[h], xsmelt = XSMELT[h];
      if (xiced <= 0.0 && xsnow > 0.0) {
        real zcflux = xsnow * 1000.0 * K.CLFSN / K.XDT;
        xsmelt = xsmelt + xsnow / K.XDT;
        XSMFLX[h] = XSMFLX[h] + zcflux;
        xcflux = xcflux - zcflux;
        xsnow = 0;
      }
      XICEC[h] = xicec;
      XSNOW[h] = xsnow;
      XSMELT[h] = xsmelt;
      XCFLUX[h] = xcflux;
      bool sea = xls < 0.5;
      real heat = sea ? xcflux : 0.0;
      // oceanstep
      real w = SS[5];
      YCLSST2[h] = (1.0 - w) * YCLSST[(int)SS[3] * NH + h] + w * YCLSST[(int)SS[4] * NH + h];
      real yls = YLS[h], yiced = XICED[h], ymld = YMLD[h], yfldo = YFLDO[h];
      real zcpsdt = K.DTMIX / (K.CRHOS * K.CPS);
      real ysst = YSST[h], zsst = ysst, yiflux = 0;
      if (yls < 1.0 && yiced <= 0.0) zsst = zsst + (heat + yfldo) * zcpsdt / ymld;
      if (yls < 1.0 && yiced > 0.0) yiflux = yiflux - yfldo - heat;
      if (ysst < K.TFREEZE && yls < 1.0) {
        yiflux = yiflux + (K.TFREEZE - zsst) * ymld / zcpsdt;
        zsst = K.TFREEZE;
      }
      if (yiced > 0.0 && yls < 1.0) {
        real zf = (K.TFREEZE - zsst) * ymld / zcpsdt;
        zsst = zsst + zf * zcpsdt / ymld;
        yiflux = yiflux + zf;
      }
      YSST[h] = zsst;
      XSST[h] = zsst;
      XMLD[h] = ymld;
      XOHEAT[h] = -yiflux;
      XOFLUX[h] = XOHEAT[h];
      if (sea) XSNDCH[h] = XSNDCH[h] + (xsnow - SNOWOLD[h]);
    } else {
      NACC[h] = NACC[h] + 1.0;
    }
    if (!(DLS[h] < 0.5)) continue;
    real dts = XTS[h], dicec = XICEC[h];
    if (coupled) {
      SEA_DSST[h] = XSST[h];
      SEA_DTS[h] = dts;
      DMLD[h] = XMLD[h];
      DICEC[h] = dicec;
      DICED[h] = XICED[h];
      DSNOW[h] = XSNOW[h];
      DSMELT[h] = XSMELT[h];
      DSNDCH[h] = XSNDCH[h];
    } else {
      CHEATA[h] = DSHFL[h] + DSWFL[NL * NH + h] + DLWFL[NL * NH + h] + DLHFL[h] + CHEATA[h];
      CPRSA[h] = DPRS[h] + CPRSA[h];
    }
    real dp = DP[h];
    DT[NL * NH + h] = dts;
    real dqs = K.RDBRV * K.RA1 * std::exp(K.RA2 * (dts - K.TMELT) / (dts - K.RA4)) / dp;
    dqs = dqs / (1.0 - (1.0 / K.RDBRV - 1.0) * dqs);
    SEA_DQS[h] = dqs;
    DQ[NL * NH + h] = dqs;
    real taux = DTAUX[h], tauy = DTAUY[h];
    real zz0 = std::max(K.CHARNOCK * std::sqrt(taux * taux + tauy * tauy) * K.GASCON * dts / (K.GA * dp), K.DZ0SEA);
    DRHS[h] = K.DRHSSEA * (1.0 - dicec) + K.DRHSICE * dicec;
    DALB[h] = K.ALBSEA * (1.0 - dicec) + dicec * std::min(K.ALBICE, 0.5 + 0.025 * (273.0 - dts));
    DSALB[h] = K.DOCEANALB1 * (1.0 - dicec) + dicec * std::min(K.DICEALBMX1, K.DICEALBMN1 + 0.025 * (273.0 - dts));
    DSALB[NH + h] = K.DOCEANALB2 * (1.0 - dicec) + dicec * std::min(K.DICEALBMX2, K.DICEALBMN2 + 0.025 * (273.0 - dts));
    DZ0[h] = zz0 * (1.0 - dicec) + K.DZ0ICE * dicec;
  }
}

// physics/carbon/wgsl/carbonstep.wgsl:1-50.
void carbon(Model& m) {
  const Consts& K = m.k;
  const int NH = m.NHOR, NL = m.NLEV;
  real *DPRC = m.F("dprc"), *DPRL = m.F("dprl"), *LP = m.F("localprecip"), *LAP = m.F("localavgprecip"),
         *CS = m.F("carbon_step"), *DT = m.F("dt"), *DLS = m.F("dls"), *CO2 = m.F("co2"), *DP = m.F("dp"),
         *LW = m.F("localweathering"), *LAT = m.F("localavgtemps"), *LAW = m.F("localavgweather");
  for (int h = 0; h < NH; ++h) {
    real precip = (DPRC[h] + DPRL[h]) * 3.154e9;
    LP[h] = precip;
    LAP[h] = LAP[h] + precip * K.TIMEWEIGHT;
    if (CS[0] == 0.0) continue;
    real tsurf = DT[NL * NH + h];
    if (K.NCARBON != 0) {
      real weathering = 0;
      if (DLS[h] > 0.5 && tsurf >= 273.15) {
        real pco2 = CO2[0] * DP[h] * 1.0e-5;
        weathering = fpow(pco2 / K.CO2EARTH, K.BETA) * std::exp(K.KACT * (tsurf - 288.0)) * fpow(precip / K.PEARTH, 0.65);
        if (K.NSUPPLY != 0) {
          real wmaxp = std::max(K.WMAX / K.VEARTH, 2.0e-15);
          weathering = wmaxp * (1.0 - std::exp(-weathering / wmaxp));
        }
      }
      LW[h] = weathering * (K.PLARAD * K.PLARAD) / (K.RAD_EARTHSQ * 0.29);
    }
    LAT[h] = LAT[h] + tsurf * K.TIMEWEIGHT;
    LAW[h] = LAW[h] + LW[h] * K.TIMEWEIGHT;
  }
}

// physics/storm/wgsl/storm.wgsl:1-208 (hurricanestep, after hurricanemod.f90):
// environmental CAPE and its neutral-buoyancy pressure, potential intensity,
// entropy deficit, absolute vorticity, ventilation, genesis potential and
// shear per column; nothing when NSTORMDIAG is 0 (storm/index.ts:27).
namespace storm_diag {
const real CPD = 1005.7, CL = 2500.0, RVP = 461.5, ALV0 = 2.501e6, CPVMCL = -630.0;
struct Cape {
  real energy, temperature, pressure;
};
real es(real tc) { return 6.112 * std::exp(17.67 * tc / (243.5 + tc)); }                       // storm.wgsl:28-30
real vapor(real r, real p, real rd) { return r * p / (rd / RVP + r); }                         // :32-35
real mixing(real e, real p, real rd) { return (rd / RVP) * e / (p - e); }                      // :37-40
real density(real t, real rt, real r, real rd) { return t * (1 + r / (rd / RVP)) / (1 + rt); }  // :42-45
real entropy(real t, real r, real p, real rd) {                                                // :47-55
  const real e = vapor(r, p, rd);
  const real rh = std::min(e / es(t - 273.15), (real)1);
  const real lv = ALV0 + CPVMCL * (t - 273.15);
  const real dry = (CPD + r * CL) * std::log(t) - rd * std::log(p - e);
  if (r == 0) return dry;
  return dry + lv * r / t - r * RVP * std::log(rh);
}
// storm.wgsl:57-126; levels 0 (top) .. n - 1 (bottom).
Cape cape(const real* st, const real* sr, const real* sp, int n, real tp, real rp, real pp, real rd) {
  if (rp < 1e-6 || tp < 200 || pp <= 0) return {0, -1, -1};
  const real rh = std::min(vapor(rp, pp, rd) / es(tp - 273.15), (real)1);
  const real parcel = entropy(tp, rp, pp, rd);
  const real plcl = pp * std::pow(rh, tp / (1669 - 122 * rh - tp));
  real b[MAXL];
  for (int l = n - 1; l >= 0; --l) {
    real tg, rg = rp;
    if (sp[l] >= plcl) {
      tg = tp * std::pow(sp[l] / pp, rd / CPD);
    } else {
      real next = st[l];
      tg = 0;
      int count = 0;
      while (!(std::fabs(next - tg) <= 0.001)) {
        tg = next;
        const real tc = tg - 273.15, enew = es(tc);
        rg = mixing(enew, sp[l], rd);
        ++count;
        const real lv = ALV0 + CPVMCL * tc;
        const real sl = (CPD + rp * CL + lv * lv * rg / (RVP * tg * tg)) / tg;
        const real em = vapor(rg, sp[l], rd);
        if (sp[l] - em <= 0 || tg <= 0) return {0, st[l], -1};
        const real sg = (CPD + rp * CL) * std::log(tg) - rd * std::log(sp[l] - em) + lv * rg / tg;
        next = tg + (count < 3 ? (real)0.3 : (real)1) * (parcel - sg) / sl;
        if (count > 500 || enew > sp[l] - 1 || !(next > 0)) return {0, st[n - 1], sp[n - 1]};
      }
    }
    b[l] = density(tg, rp, rg, rd) - density(st[l], sr[l], sr[l], rd);
  }
  int inb = n - 1;
  for (int l = 0; l < n; ++l)
    if (b[l] > 0) inb = std::min(inb, l);
  if (inb == n - 1) return {0, st[n - 1], 0};
  real area = 0;
  for (int l = n - 2; l >= inb; --l) area += rd * (b[l] + b[l + 1]) * (sp[l + 1] - sp[l]) / (sp[l] + sp[l + 1]);
  area += rd * (pp - sp[n - 1]) / (pp + sp[n - 1]) * b[n - 1];
  real tob = st[inb], lnb = sp[inb];
  if (inb > 0) {
    lnb = (sp[inb - 1] * b[inb] - sp[inb] * b[inb - 1]) / (b[inb] - b[inb - 1]);
    area += rd * b[inb] * (sp[inb] - lnb) / (sp[inb] + lnb);
    tob = (st[inb] * (lnb - sp[inb - 1]) + st[inb - 1] * (sp[inb] - lnb)) / (sp[inb] - sp[inb - 1]);
  }
  return {std::max(area, (real)0), tob, lnb};
}
real reduced(real vi, real vithresh) {  // storm.wgsl:128-133
  if (vi == 0 || std::fabs(vi) >= vithresh) return 0;
  return 2 / std::sqrt((real)3) * std::cos(std::acos(-vi / vithresh) / 3);
}
}  // namespace storm_diag

void storm(Model& m) {  // storm.wgsl:135-208
  using namespace storm_diag;
  const Consts& K = m.k;
  if (K.NSTORMDIAG <= 0) return;
  const int NH = m.NHOR, NL = m.NLEV;
  const real *DT = m.F("dt"), *DQ = m.F("dq"), *DU = m.F("du"), *DV = m.F("dv"), *GZ = m.F("gz"), *DP = m.F("dp");
  const real* sg = m.TB("sigma");
  real *CAPEN = m.F("capen"), *LNB = m.F("lnb"), *MPOTI = m.F("mpoti"), *CHIM = m.F("chim"), *LAAV = m.F("laav"),
       *VENTI = m.F("venti"), *VRMPI = m.F("vrmpi"), *GPI = m.F("gpi"), *SHEAR = m.F("shear");
  const real rd = K.GASCON;
  for (int h = 0; h < NH; ++h) {
    real st[MAXL], sr[MAXL], sp[MAXL];
    const real msl = DP[h] * 0.01, sst = DT[NL * NH + h];
    int i600 = 0, i850 = 0, i200 = 0;
    bool cold = false;
    for (int l = 0; l < NL; ++l) {
      st[l] = DT[l * NH + h];
      sr[l] = DQ[l * NH + h];
      sp[l] = msl * sg[l];
      cold = cold || st[l] <= 100;
      if (std::fabs(sg[l] - 0.6) < std::fabs(sg[i600] - 0.6)) i600 = l;
      if (std::fabs(sg[l] - 0.85) < std::fabs(sg[i850] - 0.85)) i850 = l;
      if (std::fabs(sg[l] - 0.2) < std::fabs(sg[i200] - 0.2)) i200 = l;
    }
    const int bottom = NL - 1;
    const real u8 = DU[i850 * NH + h], v8 = DV[i850 * NH + h], u2 = DU[i200 * NH + h], v2 = DV[i200 * NH + h];
    const real shear = std::fabs(std::sqrt(u2 * u2 + v2 * v2) - std::sqrt(u8 * u8 + v8 * v8));
    const real vort = GZ[i850 * NH + h] * K.WW;
    real deficit = 1;
    if (sr[i600] > 0 && sr[bottom] > 0) {
      const real smr = mixing(es(st[i600] - 273.15), sp[i600], rd);
      const real sms = entropy(st[i600], smr, sp[i600], rd);
      const real sme = entropy(st[i600], std::min(sr[i600], smr), sp[i600], rd);
      const real smb = entropy(sst, DQ[NL * NH + h], msl, rd);
      const real smo = entropy(sst, mixing(es(sst - 273.15), msl, rd), msl, rd);
      if (smo != smb) deficit = (sms - sme) / (smo - smb);
    }
    Cape env{-1, -1, -1};
    real vmax = -1;
    if (sst > 278.15 && !cold && msl > 0) {
      env = cape(st, sr, sp, NL, st[bottom], sr[bottom], sp[bottom], rd);
      real pm = 970, old = pm, next = 0, capem = 0, capems = 0, ratio = 1;
      bool failed = false;
      int count = 0;
      while (!(std::fabs(next - old) <= 0.5)) {
        const real pp = std::min(pm, (real)1000);
        const real rp = (rd / RVP) * sr[bottom] * msl / (pp * (rd / RVP + sr[bottom]) - sr[bottom] * msl);
        capem = cape(st, sr, sp, NL, st[bottom], rp, pp, rd).energy;
        const real rs = mixing(es(sst - 273.15), pp, rd);
        const Cape sat = cape(st, sr, sp, NL, sst, rs, pp, rd);
        capems = sat.energy;
        ratio = sst / sat.temperature;
        const real tvav = 0.5 * (density(st[bottom], sr[bottom], sr[bottom], rd) + density(sst, rs, rs, rd));
        const real cat = std::max((capem - env.energy) + 0.5 * K.CKCD * ratio * (capems - capem), (real)0);
        next = msl * std::exp(-cat / (rd * tvav));
        old = pm;
        pm = next;
        ++count;
        if (count > 200 || pm < 400 || !(pm > 0)) {
          failed = true;
          break;
        }
      }
      if (!failed) vmax = std::sqrt(std::max((real)0, K.CKCD * ratio * std::max((real)0, capems - capem)));
    }
    const real vi = vmax > 0 ? shear * deficit / vmax : 1;
    const real rh = vapor(sr[i600], sp[i600], rd) / es(st[i600] - 273.15);
    const real v70 = vmax / 70, damp = 1 + 0.1 * shear;
    CAPEN[h] = env.energy;
    LNB[h] = env.pressure;
    MPOTI[h] = vmax;
    CHIM[h] = deficit;
    LAAV[h] = vort;
    VENTI[h] = vi;
    VRMPI[h] = reduced(vi, K.VITHRESH);
    GPI[h] = std::pow(std::fabs(vort * 1e5), (real)1.5) * std::pow(rh * 2, (real)3) * v70 * v70 * v70 / (damp * damp);
    SHEAR[h] = shear;
  }
}

// snapshot/wgsl/pack.wgsl:1-107.
void pack(Model& m) {
  const Consts& K = m.k;
  const int NH = m.NHOR, NL = m.NLEV;
  real *SNAP = m.F("snapshot"), *TR = m.F("snapshot_tracking"), *SS = m.F("snapshot_step"), *DT = m.F("dt");
  int step = (int)SS[0], window = (int)SS[1];
  int jet = (int)K.JET;
  auto put = [&](int index, int h, real v) { SNAP[index * NH + h] = v; };
  real *DTSA = m.F("dtsa"), *DU = m.F("du"), *DV = m.F("dv"), *DCC = m.F("dcc"), *DPRC = m.F("dprc"),
         *DPRL = m.F("dprl"), *DP = m.F("dp"), *DQVI = m.F("dqvi"), *DICEC = m.F("dicec"), *DSNOW = m.F("dsnow"),
         *DWATC = m.F("dwatc"), *DALB = m.F("dalb"), *DLWFL = m.F("dlwfl"), *DLS = m.F("dls"), *DSWFL = m.F("dswfl"),
         *DSMELT = m.F("dsmelt"), *DSHFL = m.F("dshfl"), *DLHFL = m.F("dlhfl"), *DEVAP = m.F("devap"),
         *DRUNOFF = m.F("drunoff"), *DFOREST = m.F("dforest"), *DLAI = m.F("dlai"), *DPRS = m.F("dprs"),
         *DICED = m.F("diced"), *DGLAC = m.F("dglac"), *DNPP = m.F("dnpp"), *GMU0 = m.F("gmu0"), *DQ = m.F("dq");
  const char* storm[9] = {"capen", "lnb", "mpoti", "chim", "laav", "venti", "vrmpi", "gpi", "shear"};
  for (int h = 0; h < NH; ++h) {
    real t = DT[NL * NH + h];
    real* tr = TR + h;
    if (tr[7 * NH] == 0.0) {
      tr[0] = t;
      tr[NH] = t;
      tr[7 * NH] = 1.0;
    }
    tr[0] = std::min(tr[0], t);
    tr[NH] = std::max(tr[NH], t);
    if (step > 0 && step % window == 0) {
      real range = tr[NH] - tr[0];
      tr[2 * NH] = tr[0];
      tr[3 * NH] = tr[NH];
      tr[4 * NH] = range;
      tr[5 * NH] += range;
      tr[6 * NH] += 1.0;
      tr[7 * NH] = 0.0;
      tr[8 * NH] = 1.0;
    }
    if (SS[2] == 0.0) continue;
    put(0, h, DT[NL * NH + h]);
    put(1, h, DTSA[h]);
    put(2, h, DU[(NL - 1) * NH + h]);
    put(3, h, DV[(NL - 1) * NH + h]);
    put(4, h, DCC[NL * NH + h]);
    put(5, h, DPRC[h] + DPRL[h]);
    put(6, h, DP[h]);
    put(7, h, DQVI[h]);
    put(8, h, DICEC[h]);
    put(9, h, DSNOW[h]);
    put(10, h, DWATC[h]);
    put(11, h, DALB[h]);
    put(12, h, DU[jet * NH + h]);
    put(13, h, DV[jet * NH + h]);
    put(14, h, -DLWFL[h]);
    put(15, h, DLS[h]);
    put(16, h, DSWFL[h] + DLWFL[h]);
    put(17, h, DSMELT[h] * -333700000.0 + DSWFL[NL * NH + h] + DLWFL[NL * NH + h] + DSHFL[h] + DLHFL[h]);
    put(18, h, -DEVAP[h]);
    put(19, h, DRUNOFF[h]);
    put(20, h, DFOREST[h]);
    put(21, h, DLAI[h]);
    put(22, h, DPRS[h]);
    put(23, h, DSMELT[h]);
    put(24, h, DICED[h]);
    put(25, h, DGLAC[h]);
    put(27, h, DSWFL[NL * NH + h]);
    put(28, h, DLWFL[NL * NH + h]);
    put(29, h, DSHFL[h]);
    put(30, h, DLHFL[h]);
    put(31, h, DPRC[h]);
    put(32, h, DPRL[h]);
    put(33, h, DSWFL[h]);
    put(34, h, DLWFL[h]);
    bool windowed = tr[8 * NH] != 0.0;
    put(35, h, windowed ? tr[2 * NH] : tr[0]);
    put(36, h, windowed ? tr[3 * NH] : tr[NH]);
    put(37, h, windowed ? tr[4 * NH] : tr[NH] - tr[0]);
    put(38, h, tr[5 * NH]);
    put(39, h, tr[6 * NH]);
    put(40, h, DNPP[h]);
    put(41, h, GMU0[h]);
    tr[5 * NH] = 0;
    tr[6 * NH] = 0;
    for (int l = 0; l < NL; ++l) {
      int f = 51 + 5 * l;
      put(f, h, DT[l * NH + h]);
      put(f + 1, h, DU[l * NH + h]);
      put(f + 2, h, DV[l * NH + h]);
      put(f + 4, h, DCC[l * NH + h]);
    }
    for (int i = 0; i < 9; ++i) put(42 + i, h, m.F(storm[i])[h]);
    int lowest = NL - 1;
    real qsat = sat_divided(K, DT[lowest * NH + h], DP[h] * K.SIGMA_LOW);
    put(51 + 5 * lowest + 3, h, std::max(0.0, DQ[lowest * NH + h]) / std::max(1.17549435e-38, qsat));
  }
}

// ----------------------------------------------------------------- stages
void gridpointa(Model& m) {
  const int L = m.L;
  legendre_dv2uv(m, "sd", "sz", "fgu", "fgv", L, m.k.PLAVOR);
  legendre_inverse(m, "sd", "fgd", "legendre_qi", L);
  legendre_inverse(m, "st", "fgt", "legendre_qi", L);
  legendre_inverse(m, "sz", "fgz", "legendre_qi", L);
  legendre_inverse(m, "sq", "fgq", "legendre_qi", L);
  legendre_inverse(m, "sp", "fgp", "legendre_qi", 1);
  legendre_inverse(m, "sp", "fgpj", "legendre_qj", 1);
  fourier_dlambda(m, "fgp", "fgpmt", 1);
  const char* inv[9][2] = {{"fgu", "gu"}, {"fgv", "gv"}, {"fgt", "gt"}, {"fgd", "gd"}, {"fgz", "gz"},
                           {"fgpj", "gpj"}, {"fgpmt", "gpmt"}, {"fgp", "gp"}, {"fgq", "gq"}};
  for (auto& p : inv) fourier_inverse(m, p[0], p[1], m.planes(p[0]) / (m.NLAT * m.NFC));
  calcgp(m);
  const char* fw[10][2] = {{"gtn", "fgtn"}, {"gqn", "fgqn"}, {"gut", "fgut"}, {"gvt", "fgvt"}, {"guz", "fguz"},
                           {"gvz", "fgvz"}, {"gke", "fgke"}, {"gvpp", "fgvpp"}, {"guq", "fguq"}, {"gvq", "fgvq"}};
  for (auto& p : fw) fourier_forward(m, p[0], p[1], m.planes(p[0]) / m.NHOR);
  legendre_forward(m, "fgvpp", "spt", "legendre_qc", 1);
  legendre_uv2dv(m, "fgvz", "fguz", "fgke", "sdt", "szt", L);
  legendre_qtend(m, "fgut", "fgvt", "fgtn", "stt", L);
  legendre_qtend(m, "fguq", "fgvq", "fgqn", "sqt", L);
}

void physics_in_stage(Model& m) {
  const int L = m.L;
  legendre_dv2uv(m, "sd", "sz", "fgu", "fgv", L, m.k.PLAVOR);
  legendre_inverse(m, "sq", "fgq", "legendre_qi", L);
  legendre_inverse(m, "st", "fgt", "legendre_qi", L);
  legendre_inverse(m, "sp", "fgp", "legendre_qi", 1);
  fourier_inverse(m, "fgu", "gu", L);
  fourier_inverse(m, "fgv", "gv", L);
  fourier_inverse(m, "fgt", "gt", L);
  fourier_inverse(m, "fgp", "gp", 1);
  fourier_inverse(m, "fgq", "gq", L);
  physics_in(m);
}

void radiation_stage(Model& m) {
  solang(m);
  if (m.k.OZONE != 0) mko3(m);
  swr(m);
  lwr(m);
  radstep(m);
}

void precipitation_stage(Model& m) {
  legendre_inverse(m, "sqt", "fdqt", "legendre_qi", m.L);
  fourier_inverse(m, "fdqt", "dqt", m.L);
  kuo(m);
  mkdca(m);
  rain_column(m);
}

void surface_stage(Model& m) {
  soil(m);
  mkradv(m);
  land_surface(m);
  if (m.k.ICE_COUPLED != 0) sea_ice(m);
  sea(m);
}

void physics_out_stage(Model& m) {
  const int L = m.L;
  physics_out(m);
  fourier_forward(m, "gtdt", "fgtdt", L);
  fourier_forward(m, "gudt", "fgudt", L);
  fourier_forward(m, "gvdt", "fgvdt", L);
  fourier_forward(m, "gqdt", "fgqdt", L);
  legendre_forward(m, "fgtdt", "stt", "legendre_qc", L);
  legendre_forward(m, "fgqdt", "sqt", "legendre_qc", L);
  legendre_uv2dv(m, "fgudt", "fgvdt", nullptr, "sdt", "szt", L);
}

void spectrald_stage(Model& m) {
  const int L = m.L;
  spectrald_diffusion(m);
  legendre_dv2uv(m, "sdp", "szp", "fzu", "fzv", L, m.k.PLAVOR);
  fourier_inverse(m, "fzu", "zu", L);
  fourier_inverse(m, "fzv", "zv", L);
  legendre_dv2uv(m, "zdsdp1", "zdszp1", "fzdu", "fzdv", L, 0.0);
  fourier_inverse(m, "fzdu", "zdu", L);
  fourier_inverse(m, "fzdv", "zdv", L);
  mkdheat(m, 1);
  fourier_forward(m, "zdtdt", "fzdtdt", L);
  legendre_forward(m, "fzdtdt", "zstt1", "legendre_qc", L);
  legendre_dv2uv(m, "zdsdp2", "zdszp2", "fzdu", "fzdv", L, 0.0);
  fourier_inverse(m, "fzdu", "zdu", L);
  fourier_inverse(m, "fzdv", "zdv", L);
  mkdheat(m, 2);
  fourier_forward(m, "zdekin", "fzdekin", L);
  legendre_forward(m, "fzdekin", "zsdef", "legendre_qc", L);
  mean_mode(m, "zsdef");
  legendre_inverse(m, "zsdef", "fzdekin", "legendre_qi", L);
  fourier_inverse(m, "fzdekin", "zdekin", L);
  mkdheat(m, 3);
  fourier_forward(m, "zdtdt", "fzdtdt", L);
  legendre_forward(m, "fzdtdt", "zstt2", "legendre_qc", L);
  spectrald_update(m);
}

void full_step(Model& m) {
  gridpointa(m);
  spectrala(m);
  physics_in_stage(m);
  fixer(m);
  surflx(m);
  vdiff(m);
  radiation_stage(m);
  precipitation_stage(m);
  surface_stage(m);
  carbon(m);
  storm(m);
  physics_out_stage(m);
  spectrald_stage(m);
  pack(m);
}

thread_local std::string g_error;

}  // namespace

extern "C" {

const char* ora_last_error() { return g_error.c_str(); }

void* ora_create(int truncation, int levels) {
  try {
    return new Model(truncation, levels);
  } catch (const std::exception& e) {
    g_error = e.what();
    return nullptr;
  }
}

void ora_destroy(void* p) { delete static_cast<Model*>(p); }

int ora_set_const(void* p, const char* name, double value) {
  Model& m = *static_cast<Model*>(p);
#define SETC(n)                     \
  if (std::strcmp(name, #n) == 0) { \
    m.k.n = (real)value;            \
    return 0;                       \
  }
  ORACLE_CONSTS(SETC)
#undef SETC
  g_error = std::string("unknown constant ") + name;
  return -1;
}

// kind 0: state field, 1: table. Returns the element count, or -1.
long ora_size(void* p, int kind, const char* name) {
  Model& m = *static_cast<Model*>(p);
  auto& map = kind == 0 ? m.state : m.tables;
  auto it = map.find(name);
  if (it == map.end()) return -1;
  return (long)it->second.size();
}

int ora_set(void* p, int kind, const char* name, const double* values, long n) {
  Model& m = *static_cast<Model*>(p);
  if (kind == 0) {
    auto it = m.state.find(name);
    if (it == m.state.end() || (long)it->second.size() != n) {
      g_error = std::string("bad state field ") + name;
      return -1;
    }
    for (long i = 0; i < n; ++i) it->second[i] = (real)values[i];
  } else {
    Vec v((size_t)n);
    for (long i = 0; i < n; ++i) v[i] = (real)values[i];
    m.tables[name] = std::move(v);
  }
  return 0;
}

int ora_get(void* p, int kind, const char* name, double* values, long n) {
  Model& m = *static_cast<Model*>(p);
  auto& map = kind == 0 ? m.state : m.tables;
  auto it = map.find(name);
  if (it == map.end() || (long)it->second.size() != n) {
    g_error = std::string("bad field ") + name;
    return -1;
  }
  for (long i = 0; i < n; ++i) values[i] = (double)it->second[i];
  return 0;
}

// Runs one named stage (the reference's dispatch groups) or a whole step.
int ora_run(void* p, const char* stage) {
  Model& m = *static_cast<Model*>(p);
  try {
    std::string s(stage);
    if (s == "step") full_step(m);
    else if (s == "gridpointa") gridpointa(m);
    else if (s == "spectrala") spectrala(m);
    else if (s == "physics_in") physics_in_stage(m);
    else if (s == "fixer") fixer(m);
    else if (s == "surface_flux") { surflx(m); vdiff(m); }
    else if (s == "radiation") radiation_stage(m);
    else if (s == "precipitation") precipitation_stage(m);
    else if (s == "surface") surface_stage(m);
    else if (s == "carbon") carbon(m);
    else if (s == "storm") storm(m);
    else if (s == "physics_out") physics_out_stage(m);
    else if (s == "spectrald") spectrald_stage(m);
    else if (s == "pack") pack(m);
    // Single transforms on fixed fields, as the engine's kernel timer
    // launches them (the reference's verify-kernels.mjs recipe).
    else if (s == "tr_legendre_inverse") legendre_inverse(m, "st", "fgt", "legendre_qi", m.L);
    else if (s == "tr_fourier_inverse") fourier_inverse(m, "fgu", "gu", m.L);
    else if (s == "tr_fourier_forward") fourier_forward(m, "gtn", "fgtn", m.L);
    else if (s == "tr_legendre_forward") legendre_forward(m, "fgtdt", "zstt1", "legendre_qc", m.L);
    else if (s == "tr_dv2uv") legendre_dv2uv(m, "sd", "sz", "fgu", "fgv", m.L, (real)1.63299310207);
    else if (s == "tr_uv2dv") legendre_uv2dv(m, "fgvz", "fguz", "fgke", "zdsdp1", "zdszp1", m.L);
    else if (s == "tr_qtend") legendre_qtend(m, "fgut", "fgvt", "fgtn", "zstt2", m.L);
    else {
      g_error = "unknown stage " + s;
      return -1;
    }
  } catch (const std::exception& e) {
    g_error = e.what();
    return -1;
  }
  return 0;
}

}  // extern "C"
