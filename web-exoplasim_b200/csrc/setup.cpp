// Host-side FP64 set-up of one planet (configure), following the reference's
// TypeScript set-up (paths relative to src/model/climate/gcm/):
//   grid/index.ts (inigau), fourier/index.ts (tables, analyse),
//   legendre/index.ts (legini, filters, analyse), setup/pumamod/index.ts
//   (planet_ini + readnl), setup/modules/index.ts (*ini), namelist/index.ts
//   (the config's namelist edits), dynamics/setup/index.ts (initpm, initsi,
//   ludcmp/lubksb, makebm, setzt), setup/surface/index.ts (surfini, oroini),
//   setup/index.ts (constants, schedule), physics/*/index.ts (tables) and
//   calendar/** (orbit, solar position, momint).
// Everything is double precision; the engine rounds tables and state to f32
// once when it uploads them, as stepper/index.ts:110-117 does.
#include "setup.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>

namespace exogcm {

namespace {

constexpr double PI = 3.14159265359;
constexpr double TWOPI = PI + PI;
constexpr double EZ = 1.63299310207;
constexpr double RV = 461.51;
constexpr double ACPV = 1870.0;
constexpr double SBK = 5.67e-8;
constexpr int MONTHS = 14;
constexpr int SOIL = 5;

double js_round(double x) { return std::floor(x + 0.5); }
long trunc_l(double x) { return (long)std::trunc(x); }

int latitudes_for(int truncation) {
  if (truncation == 21) return 32;
  if (truncation == 42) return 64;
  if (truncation == 63) return 96;
  throw std::invalid_argument("truncation must be 21, 42 or 63");
}

// ---------------------------------------------------------------- grid
double ql(int k, double p) {  // grid/index.ts:15-30
  const double angle = std::acos(p);
  double factor = 1, sum = 0, term = 0;
  for (int j = k; j >= 0; j -= 2) {
    term = factor * std::cos(angle * j);
    sum = sum + term;
    const double z4 = (k - j + 1) * (k + j) * 0.5;
    factor = (factor * z4) / (z4 + (j - 1));
  }
  if (k % 2 == 0) sum = sum - 0.5 * term;
  double norm = std::sqrt(2.0);
  for (int j = 1; j <= k; ++j) norm = norm * std::sqrt(1 - 0.25 / ((double)j * j));
  return norm * sum;
}

void gaussian(int count, Vec& sines, Vec& weights) {  // grid/index.ts:32-63 (inigau)
  const double ipi = 3.14159265358979;
  sines.assign(count, 0);
  weights.assign(count, 0);
  const double z0 = ipi / (2 * count + 1), z1 = 1.0 / ((double)count * count * 8), z4 = 2.0 / ((double)count * count);
  for (int root = 0; root < count / 2; ++root) {
    const double guess = z0 * (2 * (root + 1) - 0.5);
    double x = std::cos(guess + z1 / std::tan(guess));
    for (int it = 0; it < 50; ++it) {
      const double value = ql(count, x);
      const double z = x * value - std::sqrt((double)(count + count + 1) / (count + count - 1)) * ql(count - 1, x);
      const double step = value * ((x * x - 1) / (count * z));
      x = x - step;
      if (std::fabs(step) < 1e-16) break;
    }
    const double z5 = ql(count - 1, x) / std::sqrt(count - 0.5);
    const double w = (z4 * (1 - x * x)) / (z5 * z5);
    sines[root] = x;
    sines[count - 1 - root] = -x;
    weights[root] = w;
    weights[count - 1 - root] = w;
  }
}

// ---------------------------------------------------------------- legendre
// legendre/index.ts:29-108 (legini): the eight tables [lat][mode].
std::map<std::string, Vec> legini(const Vec& sines, const Vec& weights, int T) {
  const int nlat = (int)sines.size();
  const int modes = (T + 1) * (T + 2) / 2;
  std::map<std::string, Vec> out;
  for (const char* k : {"qi", "qj", "qc", "qe", "qm", "qq", "qu", "qv"}) out[k] = Vec((size_t)nlat * modes, 0);
  Vec &qi = out["qi"], &qj = out["qj"], &qc = out["qc"], &qe = out["qe"], &qm = out["qm"], &qq = out["qq"],
      &qu = out["qu"], &qv = out["qv"];
  Vec pli(modes + 1, 0), pld(modes + 1, 0);
  for (int lat = 0; lat < nlat; ++lat) {
    const double sin = sines[lat], weight = weights[lat];
    const double cos2 = 1 - sin * sin, wocs = weight / cos2;
    double f1m = std::sqrt(1.5);
    pli[1] = std::sqrt(0.5);
    pli[2] = f1m * sin;
    pld[1] = 0;
    int lm = 2;
    for (int m = 0; m <= T; ++m) {
      if (m > 0) {
        lm++;
        const double f2m = -f1m * std::sqrt(cos2 / (m + m));
        f1m = f2m * std::sqrt((double)(m + m + 3));
        pli[lm] = f2m;
        if (lm < modes) {
          lm++;
          pli[lm] = f1m * sin;
          pld[lm - 1] = -m * f2m * sin;
        }
      }
      const double m2 = (double)m * m;
      for (int n = m + 2; n <= T; ++n) {
        lm++;
        const double z1 = std::sqrt(((double)(n - 1) * (n - 1) - m2) / (4.0 * (n - 1) * (n - 1) - 1));
        const double z2 = sin * pli[lm - 1] - z1 * pli[lm - 2];
        pli[lm] = z2 * std::sqrt((4.0 * n * n - 1) / ((double)n * n - m2));
        pld[lm - 1] = (1 - n) * z2 + n * z1 * pli[lm - 2];
      }
      if (lm < modes) {
        const double z3 = std::sqrt(((double)T * T - m2) / (4.0 * T * T - 1));
        pld[lm] = -T * sin * pli[lm] + (T + T + 1) * pli[lm - 1] * z3;
      } else {
        pld[lm] = -T * sin * pli[lm];
      }
    }
    int w = 0;
    for (int m = 0; m <= T; ++m)
      for (int n = m; n <= T; ++n) {
        const double invdeg = n > 0 ? 1.0 / ((double)n * (n + 1)) : 0.0;
        const size_t at = (size_t)lat * modes + w;
        const double p = pli[w + 1], d = pld[w + 1];
        qi[at] = p;
        qj[at] = d;
        qc[at] = p * weight;
        qu[at] = p * invdeg * m;
        qv[at] = d * invdeg;
        qe[at] = d * wocs;
        qq[at] = p * wocs * n * (n + 1) * 0.5;
        qm[at] = p * wocs * m;
        w++;
      }
  }
  return out;
}

// legendre/index.ts:111-136 (filters).
void filters(int T, int nfilter, int ngpt, int nspv, double kappa, double exponent, double n0, Vec& g2s,
             Vec& s2g) {
  g2s.assign(T + 1, 0);
  s2g.assign(T + 1, 0);
  for (int degree = 0; degree <= T; ++degree) {
    const double n = degree + 1;
    double shape = 1;
    switch (nfilter) {
      case 0: shape = 1; break;
      case 1: shape = 1 - n / (T + 1); break;
      case 2: shape = std::exp(-kappa * std::pow(n / T, exponent)); break;
      case 3: shape = std::exp(-std::pow((n * (n + 1)) / (n0 * (n0 + 1)), 2)); break;
      case 4: shape = std::pow(1 - n / (T + 1), 2); break;
      default: throw std::invalid_argument("filter kind must be 0-4");
    }
    g2s[degree] = 1 - ngpt + ngpt * shape;
    s2g[degree] = 1 - nspv + nspv * shape;
  }
}

// fourier/index.ts:95-115 then legendre/index.ts:334-361 (analyse): grid -> spectral in f64.
Vec analyse(const SharedSetup& sh, const double* grid) {
  const int T = sh.truncation, nlat = sh.nlat, nlon = sh.nlon, nfc = 2 * (T + 1);
  const int modes = (T + 1) * (T + 2) / 2;
  Vec four((size_t)nlat * nfc, 0);
  // Each coefficient sums the longitudes in order j = 0, 1, ...; the loop
  // over coefficients is innermost so the table rows are read contiguously.
  for (int row = 0; row < nlat; ++row) {
    double* out = &four[(size_t)row * nfc];
    for (int j = 0; j < nlon; ++j) {
      const double g = grid[(size_t)row * nlon + j];
      const double* f = &sh.fwd[(size_t)j * nfc];
      for (int c = 0; c < nfc; ++c) out[c] += g * f[c];
    }
  }
  Vec sp(2 * modes, 0);
  for (int l = 0; l < nlat / 2; ++l) {
    const double* north = &four[(size_t)l * nfc];
    const double* south = &four[(size_t)(nlat - 1 - l) * nfc];
    int w = 0;
    for (int m = 0; m <= T; ++m)
      for (int n = m; n <= T; ++n) {
        const double sign = (m + n) % 2 == 0 ? 1 : -1;
        const double weight = sh.qc_unfiltered[(size_t)l * modes + w];
        for (int part = 0; part < 2; ++part) {
          const double row = north[2 * m + part] + sign * south[2 * m + part];
          sp[2 * w + part] = sp[2 * w + part] + weight * row * sh.g2s[n];
        }
        w++;
      }
  }
  return sp;
}

// `planes` grids [plane][points] -> spectra [plane][2 * modes], on the set-up
// device when there is one.
Vec analyse_planes(const SharedSetup& sh, const double* grids, int planes, SetupDevice* device) {
  const int modes = (sh.truncation + 1) * (sh.truncation + 2) / 2;
  const size_t points = (size_t)sh.nlat * sh.nlon;
  Vec out((size_t)planes * 2 * modes);
  if (device) {
    device->analyse(sh, grids, planes, out.data());
    return out;
  }
  for (int p = 0; p < planes; ++p) {
    const Vec sp = analyse(sh, grids + p * points);
    std::copy(sp.begin(), sp.end(), out.begin() + (size_t)p * 2 * modes);
  }
  return out;
}

// ---------------------------------------------------------------- calendar
const int MONTH_DAYS[12] = {31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};
bool leap(long y) { return y % 4 == 0 && (y % 100 != 0 || y % 400 == 0); }
long year_start(long y) {
  return 365 * y + (long)std::floor((y + 3) / 4.0) - (long)std::floor((y + 99) / 100.0) +
         (long)std::floor((y + 399) / 400.0);
}
int month_days(long y, int m) { return MONTH_DAYS[m - 1] + (m == 2 && leap(y) ? 1 : 0); }

// calendar/date/index.ts:30-41 (startStep).
long start_step(long mtspd, long year, int month, long dpy, long dpm) {
  if (dpy != 365) return mtspd * (year * dpy + (month - 1) * dpm);
  long days = year_start(year);
  for (int at = 1; at < month; ++at) days += month_days(year, at);
  return mtspd * days;
}

struct Date {
  long year;
  int month, day, hour, minute;
};

// calendar/date/index.ts:43-80 (date).
Date cal_date(long step, long spd, long dpy, double step_minutes) {
  if (dpy == 365) {
    const long days = step / spd;
    long year = trunc_l(days / 365.2425);
    while (year_start(year) > days) year--;
    while (year_start(year + 1) <= days) year++;
    long day = days - year_start(year) + 1;
    int month = 1;
    while (day > month_days(year, month)) {
      day -= month_days(year, month);
      month++;
    }
    const long minutes = trunc_l(((double)(step % spd) * 1440) / spd);
    return {year, month, (int)day, (int)(minutes / 60), (int)(minutes % 60)};
  }
  const long mtspd = trunc_l((double)(dpy * spd) / 360);
  const long days = step / mtspd;
  const long doy = days % 360;
  const long minutes = trunc_l((double)(step % mtspd) * js_round(step_minutes));
  return {days / 360 + 1, (int)(doy / 30) + 1, (int)(doy % 30) + 1, (int)(minutes / 60), (int)(minutes % 60)};
}

// calendar/date/index.ts:82-112 (monthInterpolation: momint).
void month_interp(long step, long spd, long dpy, long dpm, double step_minutes, double solar_day, double out[3]) {
  const Date d = cal_date(step, spd, dpy, step_minutes);
  const double fday = d.day + ((d.hour * 60.0 + d.minute) * 60) / solar_day;
  const double current = dpy == 365 ? month_days(d.year, d.month) : (double)dpm;
  const double median = 0.5 * (current + 1);
  const int neighbour = fday > median ? d.month + 1 : d.month - 1;
  const double adjacent = dpy == 365 ? month_days(d.year, ((neighbour + 11) % 12) + 1) : (double)dpm;
  out[0] = d.month;
  out[1] = neighbour;
  out[2] = std::fabs(fday - median) / (median + 0.5 * (adjacent + 1) - 1);
}

// ---------------------------------------------------------------- namelists
// pumamod's values after planet_ini and readnl (setup/pumamod/index.ts:94-237)
// for the namelists the configuration produces: public/gcm/t*/namelists.json's
// values with GCM_NAMELIST.edits applied (namelist/index.ts:40-182).
struct Pumamod {
  double ga, gascon, akap, alr, ra1, ra2, ra4, pnu, plarad, rotspd, gsol0, eccen, mvelp, obliq, meananom0;
  int nfixorb, ngenkeplerian;
  double sidereal_year;
  double day_24hr, solar_day, sidereal_day, ww, acpd, adv, cv, ct, pnu21, rdbrv, tmelt, alv, als, psurf, plavor;
  double mpstep;
  long mtspd, ntspd, nafter, n_steps_per_year, n_days_per_year, n_start_year, n_start_step, n_days_per_month,
      m_days_per_year;
  int nkits, ndheat, nveg, nhdiff, nfilter, ngptfilter, nspvfilter;
  double filterkappa, nfilterexp, landhoskn0, dtep, dtns, dtrop, dttrp, dttl, fixedlon, tgr;
  std::vector<double> ndel, tdissd, tdissz, tdisst, tdissq, restim, t0, tfrc;
};

Pumamod pumamod(const exogcm_planet& p) {
  Pumamod pm{};
  const int T = p.truncation, L = p.levels;
  // planet_namelist: p_earth.f90 defaults, namelists.json, then the edits.
  pm.eccen = p.eccentricity;
  pm.mvelp = 102.7;
  pm.obliq = p.obliquity_deg;
  pm.rotspd = p.rotation_period_days != 1 ? 1 / p.rotation_period_days : 1.0;
  pm.sidereal_year = p.year_days * 86400.0;
  pm.meananom0 = -2.9589;
  pm.akap = 0.286;
  pm.alr = 0.0065;
  pm.gascon = p.gas_constant;
  pm.ra1 = 610.78;
  pm.ra2 = 17.2693882;
  pm.ra4 = 35.86;
  pm.pnu = 0.1;
  pm.ga = p.gravity;
  pm.plarad = p.radius_earth * 6371220.0;
  pm.gsol0 = p.flux;
  pm.nfixorb = p.fixed_orbit ? 1 : 0;
  pm.ngenkeplerian = p.keplerian ? 1 : 0;
  const double day24 = 86400.0;
  // plasim_namelist: plasimmod defaults, resolution defaults, namelists.json, edits.
  long ndpy = (long)js_round(p.year_days);
  if (p.rotation_period_days != 1)
    ndpy = std::max<long>((long)std::floor(p.year_days / p.rotation_period_days / 12 + 0.5), 1) * 12;
  const long n_start_year = ndpy == 365 ? 1 : 0;
  const double mpstep_nl = p.timestep_minutes;
  const long nstpw = (long)std::floor(7200 / p.timestep_minutes);
  pm.nkits = 3;
  pm.ndheat = 1;
  pm.nveg = p.vegetation;
  pm.nhdiff = T == 42 ? 16 : 15;
  pm.ndel.assign(L, T == 42 ? 4 : 2);
  pm.tdissq.assign(L, T == 42 ? 0.1 * day24 : 0.1);
  pm.tdisst.assign(L, T == 42 ? 0.76 * day24 : 5.6);
  pm.tdissz.assign(L, T == 42 ? 0.3 * day24 : 1.1);
  pm.tdissd.assign(L, T == 42 ? 0.06 * day24 : 0.2);
  pm.restim.assign(L, 0.0);
  pm.t0.assign(L, 250.0);
  pm.tfrc.assign(L, 0.0);
  if (L == 10) {
    pm.tfrc[0] = 20 * day24;
    pm.tfrc[1] = 100 * day24;
  }
  pm.nfilter = p.filter_kind;
  pm.ngptfilter = p.filter_gp;
  pm.nspvfilter = p.filter_sp;
  pm.filterkappa = 8;
  pm.nfilterexp = 8;
  pm.landhoskn0 = 15;
  pm.dtep = 0;
  pm.dtns = 0;
  pm.dtrop = 12000;
  pm.dttrp = 2;
  pm.dttl = 0;
  pm.fixedlon = p.substellar_longitude_deg;
  pm.tgr = 288;
  const double psurf_nl = p.pressure_bar * 1e5;
  double solar_day = day24;
  double sidereal_day = (solar_day * (ndpy - 1)) / ndpy;
  if (pm.rotspd != 1) {
    sidereal_day = day24 / pm.rotspd;
    solar_day = ndpy != 1 ? (sidereal_day * ndpy) / (ndpy - 1) : sidereal_day;
  }
  const long mdpy = (long)js_round((ndpy * sidereal_day) / day24);
  pm.day_24hr = day24;
  pm.solar_day = solar_day;
  pm.sidereal_day = sidereal_day;
  pm.ww = TWOPI / sidereal_day;
  pm.acpd = pm.gascon / pm.akap;
  pm.adv = ACPV / pm.acpd - 1;
  pm.cv = pm.plarad * pm.ww;
  pm.ct = (pm.cv * pm.cv) / pm.gascon;
  pm.pnu21 = 1 - 2 * pm.pnu;
  pm.rdbrv = pm.gascon / RV;
  pm.tmelt = 273.16;
  pm.alv = 2.5008e6;
  pm.als = 2.8345e6;
  pm.psurf = psurf_nl;
  pm.plavor = EZ;
  double mpstep = mpstep_nl;
  long mtspd = 0;
  if (mpstep > 0) {
    mtspd = trunc_l(js_round(day24) / js_round(mpstep * 60));
    mtspd = mtspd + (mtspd % 2);
  }
  if (mtspd <= 0) throw std::invalid_argument("timestep too long");
  mpstep = day24 / (mtspd * 60.0);
  pm.mpstep = mpstep;
  pm.mtspd = mtspd;
  pm.ntspd = trunc_l(js_round(solar_day) / js_round(mpstep * 60));
  pm.nafter = nstpw > 0 ? nstpw : mtspd;  // nlowio = 1 in namelists.json
  pm.n_steps_per_year = (long)js_round(pm.sidereal_year / (mpstep * 60));
  pm.n_days_per_year = ndpy;
  pm.n_start_year = n_start_year;
  pm.n_days_per_month = mdpy / 12;
  pm.m_days_per_year = mdpy;
  pm.n_start_step = start_step(mtspd, n_start_year, 1, ndpy, pm.n_days_per_month);
  return pm;
}

// ---------------------------------------------------------------- dynamics set-up
struct Dyn {
  Vec sigmah, sigma, dsigma, rdsig, damp, tfrc, tdissd, tdissz, tdisst, tdissq, sak, nindex, t0, tkp, t01s2, g, c,
      tau;
  double dtns, dtep, dttrp;
};

Vec rate(const Vec& values, double threshold, double day) {  // dayseccheck then time scale -> rate
  const double largest = *std::max_element(values.begin(), values.end());
  Vec out(values.size());
  for (size_t i = 0; i < values.size(); ++i) {
    double v = (largest < threshold && largest > 0) ? values[i] * day : values[i];
    out[i] = v > 0 ? day / (TWOPI * v) : 0;
  }
  return out;
}

// dynamics/setup/index.ts:27-152 (initpm for NEQSIG = 0, initsi).
Dyn initpm(int T, int L, const Pumamod& pm, double akap) {
  Dyn s;
  s.sigmah.resize(L);
  for (int l = 0; l < L; ++l) {
    const double z = (l + 1.0) / L;
    s.sigmah[l] = 0.75 * z + 1.75 * z * z * z - 1.5 * z * z * z * z;
  }
  s.dsigma.resize(L);
  s.rdsig.resize(L);
  s.sigma.resize(L);
  for (int l = 0; l < L; ++l) {
    s.dsigma[l] = l == 0 ? s.sigmah[0] : s.sigmah[l] - s.sigmah[l - 1];
    s.rdsig[l] = 0.5 / s.dsigma[l];
    s.sigma[l] = l == 0 ? 0.5 * s.sigmah[0] : 0.5 * (s.sigmah[l - 1] + s.sigmah[l]);
  }
  const double day = pm.day_24hr, threshold = day / pm.mtspd;
  s.damp = rate(pm.restim, threshold, day);
  s.tfrc = rate(pm.tfrc, threshold, day);
  s.tdissd = rate(pm.tdissd, threshold, day);
  s.tdissz = rate(pm.tdissz, threshold, day);
  s.tdisst = rate(pm.tdisst, threshold, day);
  s.tdissq = rate(pm.tdissq, threshold, day);
  const int nrsp = (T + 1) * (T + 2);
  s.sak.assign((size_t)L * nrsp, 0);
  for (int l = 0; l < L; ++l) {
    const double power = pm.ndel[l];
    const double scale = 1.0 / std::pow((double)(T - pm.nhdiff), power);
    int r = 0;
    for (int m = 0; m <= T; ++m)
      for (int n = m; n <= T; ++n) {
        const double v = n >= pm.nhdiff ? scale * std::pow((double)(n - pm.nhdiff), power) : 0.0;
        s.sak[(size_t)l * nrsp + r] = v;
        s.sak[(size_t)l * nrsp + r + 1] = v;
        r += 2;
      }
  }
  s.nindex.assign(nrsp, 0);
  {
    int r = 0;
    for (int m = 0; m <= T; ++m)
      for (int n = m; n <= T; ++n) {
        s.nindex[r] = s.nindex[r + 1] = n;
        r += 2;
      }
  }
  s.t0.resize(L);
  for (int l = 0; l < L; ++l) s.t0[l] = pm.t0[l] / pm.ct;
  s.dtns = pm.dtns / pm.ct;
  s.dtep = pm.dtep / pm.ct;
  s.dttrp = pm.dttrp / pm.ct;
  // initsi
  const int n = L;
  auto at = [n](int i, int j) { return (size_t)j * n + i; };
  s.tkp.resize(n);
  s.t01s2.assign(n, 0);
  s.g.assign(n * n, 0);
  s.c.assign(n * n, 0);
  s.tau.assign(n * n, 0);
  for (int l = 0; l < n; ++l) s.tkp[l] = akap * s.t0[l];
  for (int l = 0; l < n - 1; ++l) s.t01s2[l] = s.t0[l + 1] - s.t0[l];
  Vec alp(n, 0);
  for (int l = 1; l < n; ++l) alp[l] = std::log(s.sigmah[l]) - std::log(s.sigmah[l - 1]);
  s.g[at(0, 0)] = 1;
  for (int l = 1; l < n; ++l) {
    s.g[at(l, l)] = 1 - (alp[l] * s.sigmah[l - 1]) / s.dsigma[l];
    for (int k = 0; k < l; ++k) s.g[at(l, k)] = alp[l];
  }
  for (int l = 0; l < n; ++l)
    for (int k = 0; k < n; ++k) s.c[at(l, k)] = s.g[at(k, l)] * (s.dsigma[l] / s.dsigma[k]);
  double t01 = s.t01s2[0], sig = s.sigmah[0];
  s.tau[at(0, 0)] = 0.5 * t01 * (sig - 1) + s.tkp[0];
  for (int k = 1; k < n; ++k) s.tau[at(k, 0)] = 0.5 * t01 * s.dsigma[k];
  for (int l = 1; l < n; ++l) {
    const double pt01 = t01, psig = sig;
    t01 = s.t01s2[l];
    sig = s.sigmah[l];
    for (int k = 0; k < n; ++k) {
      const int below = k <= l ? 1 : 0, above = k < l ? 1 : 0;
      double value = pt01 * (psig - above);
      if (l < n - 1) value = value + t01 * (sig - below);
      value = value * s.rdsig[l] * s.dsigma[k];
      if (k <= l) value = value + s.tkp[l] * s.c[at(k, l)];
      s.tau[at(k, l)] = value;
    }
  }
  return s;
}

// dynamics/setup/index.ts:154-211 (ludcmp + lubksb with partial pivoting).
Vec invert(Vec a, int n) {
  auto at = [n](int i, int j) { return (size_t)j * n + i; };
  Vec scale(n);
  for (int i = 0; i < n; ++i) {
    double largest = 0;
    for (int j = 0; j < n; ++j) largest = std::max(largest, std::fabs(a[at(i, j)]));
    scale[i] = 1 / largest;
  }
  std::vector<int> index(n);
  for (int j = 0; j < n; ++j) {
    for (int i = 1; i < j; ++i) {
      double dot = 0;
      for (int k = 0; k < i; ++k) dot += a[at(i, k)] * a[at(k, j)];
      a[at(i, j)] -= dot;
    }
    double largest = 0;
    int pivot = j;
    for (int i = j; i < n; ++i) {
      if (j > 0) {
        double dot = 0;
        for (int k = 0; k < j; ++k) dot += a[at(i, k)] * a[at(k, j)];
        a[at(i, j)] -= dot;
      }
      const double size = scale[i] * std::fabs(a[at(i, j)]);
      if (size >= largest) {
        pivot = i;
        largest = size;
      }
    }
    if (j != pivot) {
      for (int k = 0; k < n; ++k) std::swap(a[at(pivot, k)], a[at(j, k)]);
      scale[pivot] = scale[j];
    }
    index[j] = pivot;
    if (a[at(j, j)] == 0) a[at(j, j)] = 5e-324;
    for (int i = j + 1; i < n; ++i) a[at(i, j)] /= a[at(j, j)];
  }
  Vec inverse((size_t)n * n);
  for (int column = 0; column < n; ++column) {
    Vec b(n, 0);
    b[column] = 1;
    int first = -1;
    for (int i = 0; i < n; ++i) {
      const int li = index[i];
      double sum = b[li];
      b[li] = b[i];
      if (first >= 0) {
        for (int j = first; j < i; ++j) sum -= a[at(i, j)] * b[j];
      } else if (sum != 0) {
        first = i;
      }
      b[i] = sum;
    }
    for (int i = n - 1; i >= 0; --i) {
      double sum = b[i];
      for (int j = i + 1; j < n; ++j) sum -= a[at(i, j)] * b[j];
      b[i] = sum / a[at(i, i)];
    }
    std::copy(b.begin(), b.end(), inverse.begin() + (size_t)column * n);
  }
  return inverse;
}

// dynamics/setup/index.ts:213-239 (makebm): the matrix before the
// diagonal term 1 / (n (n + 1)), then the inverse of each degree's.
Vec makebm_base(const Dyn& s, double delt) {
  const int n = (int)s.t0.size();
  const double d2 = delt * delt;
  Vec base((size_t)n * n);
  for (int l1 = 0; l1 < n; ++l1)
    for (int l2 = 0; l2 < n; ++l2) {
      double dot = 0;
      for (int k = 0; k < n; ++k) dot += s.g[(size_t)l1 * n + k] * s.tau[(size_t)k * n + l2];
      base[(size_t)l1 * n + l2] = d2 * (s.t0[l1] * s.dsigma[l2] + dot);
    }
  return base;
}

Vec makebm(const Vec& base, int n, int T) {
  Vec bm1((size_t)n * n * T);
  for (int degree = 1; degree <= T; ++degree) {
    Vec mat = base;
    for (int l = 0; l < n; ++l) mat[(size_t)l * n + l] += 1.0 / ((double)degree * (degree + 1));
    Vec inv = invert(mat, n);
    std::copy(inv.begin(), inv.end(), bm1.begin() + (size_t)(degree - 1) * n * n);
  }
  return bm1;
}

// dynamics/setup/index.ts:256-313 (setzt).
Vec setzt(const Dyn& s, int T, const Pumamod& pm) {
  const int L = (int)s.sigma.size();
  const double gascon = pm.gascon, ga = pm.ga, ct = pm.ct, alr = pm.alr, tgr = pm.tgr, dtrop = pm.dtrop;
  const double dttrp = s.dttrp * ct;
  auto profile = [&](double height) {
    return tgr - dtrop * alr + std::sqrt(std::pow(0.5 * alr * (height - dtrop), 2) + dttrp * dttrp) -
           0.5 * alr * (height - dtrop);
  };
  Vec trs(L);
  double sp = 1, tp = tgr, zp = 0;
  for (int l = L - 1; l >= 0; --l) {
    const double lr = std::log(sp / s.sigma[l]);
    const double first = profile(zp + ((gascon * tp) / ga) * lr);
    const double t = profile(zp + ((gascon * (0.5 * (tp + first))) / ga) * lr);
    trs[l] = t;
    zp = zp + ((0.5 * (t + tp) * gascon) / ga) * lr;
    tp = t;
    sp = s.sigma[l];
  }
  const double tropopause = std::pow((tgr - dtrop * alr) / tgr, ga / (alr * gascon));
  const double substellar = (1 / 3.463843223261725 / ct) * pm.dttl;
  const double subst1 = -substellar * std::cos((pm.fixedlon * PI) / 180);
  const double subst2 = substellar * std::sin((pm.fixedlon * PI) / 180);
  const int nrsp = (T + 1) * (T + 2), sas = 2 * (T + 1);
  Vec sr((size_t)L * nrsp, 0);
  for (int l = 0; l < L; ++l) {
    const double fac = std::max(std::sin((0.5 * PI * (s.sigma[l] - tropopause)) / (1 - tropopause)), 0.0);
    double* r = &sr[(size_t)l * nrsp];
    r[0] = std::sqrt(2.0) * (trs[l] / ct - s.t0[l]);
    r[2] = (1 / std::sqrt(6.0)) * s.dtns * fac;
    r[4] = (-2.0 / 3.0) * std::sqrt(0.4) * s.dtep * fac;
    r[sas] = subst1 * fac;
    r[sas + 1] = subst2 * fac;
  }
  return sr;
}

// ---------------------------------------------------------------- surface set-up
// get_surf_array (setup/surface/index.ts:72-103): 1 or 12 fields -> `months`.
Vec surf_field(const double* data, int found, int points, int months, double fallback) {
  Vec out((size_t)months * points, fallback);
  if (!data) return out;
  if (found < 1) throw std::invalid_argument("surface field needs at least one month");
  const int take = std::min(found, months);
  for (int i = 0; i < take * points; ++i) out[i] = data[i];
  if (take == months) return out;
  auto row = [&](int m) { return out.begin() + (size_t)m * points; };
  if (take == 12 && months == MONTHS) {
    for (int m = 12; m >= 1; --m) std::copy(row(m - 1), row(m - 1) + points, row(m));
    std::copy(row(1), row(1) + points, row(13));
    std::copy(row(12), row(12) + points, row(0));
  } else if (take == 1 && months == MONTHS) {
    for (int m = 1; m < MONTHS; ++m) std::copy(row(0), row(0) + points, row(m));
  } else {
    throw std::invalid_argument("surface climatology must have 1 or 12 fields");
  }
  return out;
}

Vec monthly(const Vec& table, long step, const Pumamod& pm, int points) {
  double mi[3];
  month_interp(step, pm.ntspd, pm.n_days_per_year, pm.n_days_per_month, pm.mpstep, pm.solar_day, mi);
  const int a = (int)mi[0], b = (int)mi[1];
  Vec out(points);
  for (int h = 0; h < points; ++h)
    out[h] = (1 - mi[2]) * table[(size_t)a * points + h] + mi[2] * table[(size_t)b * points + h];
  return out;
}

double saturation(double t, const Pumamod& pm) {  // setup/surface/index.ts:159-167
  const double q = (pm.rdbrv * pm.ra1 * std::exp((pm.ra2 * (t - pm.tmelt)) / (t - pm.ra4))) / pm.psurf;
  return q / (1 - (1 / pm.rdbrv - 1) * q);
}

double glacier_albedo(double mx, double mn, double ts, double tmelt) {
  return std::max(mn, std::min(mx, mx - ((mx - mn) * (ts - 263.16)) / (tmelt - 263.16)));
}

// oroini (setup/surface/index.ts:170-236): river directions and velocities.
void runoff(const Vec& oro, const Vec& mask, int nlat, int nlon, const Vec& sines, const Pumamod& pm, Vec& du,
            Vec& dv) {
  const int points = nlat * nlon;
  du.assign(points, 0);
  dv.assign(points, 0);
  Vec height(points);
  for (int h = 0; h < points; ++h) height[h] = mask[h] < 1 ? mask[h] - 1 : std::max(oro[h], 0.0);
  const double hmax = *std::max_element(height.begin(), height.end());
  const double hmin = *std::min_element(height.begin(), height.end());
  if ((hmax - hmin) / pm.ga <= 0.01) return;
  bool raised = true;
  Vec next(points);
  while (raised) {
    raised = false;
    for (int h = 0; h < points; ++h) {
      const int lon = h % nlon, lat = h / nlon;
      double around[4];
      int na = 0;
      around[na++] = height[lat * nlon + (lon + 1) % nlon];
      around[na++] = height[lat * nlon + (lon + nlon - 1) % nlon];
      if (lat > 0) around[na++] = height[h - nlon];
      if (lat < nlat - 1) around[na++] = height[h + nlon];
      bool lowest = true;
      double mn = around[0];
      for (int i = 0; i < na; ++i) {
        if (!(height[h] <= around[i])) lowest = false;
        mn = std::min(mn, around[i]);
      }
      if (mask[h] > 0 && lowest) {
        next[h] = 1 + mn;
        raised = true;
      } else {
        next[h] = height[h];
      }
    }
    height.swap(next);
  }
  auto rate_of = [](double slope, double spacing, double sign) {
    return ((sign * 4.2) / spacing) * std::pow(std::fabs(slope), 0.18);
  };
  for (int lat = 0; lat < nlat; ++lat) {
    const double dx = (TWOPI * std::cos(std::asin(sines[lat])) * pm.plarad) / nlon;
    for (int lon = 0; lon < nlon; ++lon) {
      const int h = lat * nlon + lon;
      const double slope = (height[lat * nlon + (lon + 1) % nlon] - height[h]) / dx;
      du[h] = rate_of(slope, dx, slope > 0 ? -1 : 1);
    }
  }
  for (int lat = 0; lat < nlat - 1; ++lat) {
    const double dy = (std::asin(sines[lat + 1]) - std::asin(sines[lat])) * pm.plarad;
    for (int lon = 0; lon < nlon; ++lon) {
      const int h = lat * nlon + lon;
      const double slope = (height[h + nlon] - height[h]) / dy;
      dv[h] = rate_of(slope, dy, slope < 0 ? -1 : 1);
    }
  }
}

// make_ice_thickness (setup/surface/index.ts:239-261).
Vec ice_thickness(const Vec& cover, int nlat, int nlon) {
  static const double factor[14] = {0.912, 0.942, 1, 1.058, 1.124, 1.161, 1.175,
                                    1.058, 0.931, 0.883, 0.88, 0.876, 0.912, 0.942};
  const int points = nlat * nlon;
  Vec out(cover.size(), 0);
  for (int month = 0; month < MONTHS; ++month)
    for (int h = 0; h < points; ++h) {
      const double c = cover[(size_t)month * points + h];
      const bool north = (h / nlon) < nlat / 2.0;
      double d = 0;
      if (north) {
        const double f = factor[month];
        if (c >= 0.9) d = 3.0 * f;
        else if (c >= 0.1) d = (0.25 + ((3.0 - 0.25) * (c - 0.1)) / (0.9 - 0.1)) * f;
        else if (c > 0) d = 0.25 * f;
      } else if (c >= 0.25) {
        d = 0.5;
      } else if (c > 0) {
        d = 0.25 + c;
      }
      out[(size_t)month * points + h] = d;
    }
  return out;
}

}  // namespace

SharedSetup build_shared(int truncation, int filter_kind, int filter_gp, int filter_sp, SetupDevice* device) {
  SharedSetup sh;
  sh.truncation = truncation;
  sh.nlat = latitudes_for(truncation);
  sh.nlon = 2 * sh.nlat;
  gaussian(sh.nlat, sh.sines, sh.weights);
  const int nfc = 2 * (truncation + 1);
  sh.fwd.assign((size_t)sh.nlon * nfc, 0);
  sh.inv.assign((size_t)nfc * sh.nlon, 0);
  for (int j = 0; j < sh.nlon; ++j) {  // fourier/index.ts:19-36
    const double lam = (2 * M_PI * j) / sh.nlon;
    for (int m = 0; m <= truncation; ++m) {
      const double c = std::cos(m * lam), s = std::sin(m * lam);
      sh.fwd[(size_t)j * nfc + 2 * m] = c / sh.nlon;
      sh.fwd[(size_t)j * nfc + 2 * m + 1] = -s / sh.nlon;
      const double weight = m == 0 ? 1 : 2;
      sh.inv[(size_t)(2 * m) * sh.nlon + j] = weight * c;
      sh.inv[(size_t)(2 * m + 1) * sh.nlon + j] = m == 0 ? 0 : -weight * s;
    }
  }
  filters(truncation, filter_kind, filter_gp, filter_sp, 8, 8, 15, sh.g2s, sh.s2g);
  if (device) {
    device->legini(sh.sines, sh.weights, truncation, sh.g2s, sh.s2g, sh.q, sh.qc_unfiltered);
    return sh;
  }
  auto tabs = legini(sh.sines, sh.weights, truncation);
  sh.qc_unfiltered = tabs["qc"];
  const int modes = (truncation + 1) * (truncation + 2) / 2;
  std::vector<int> nof(modes);
  {
    int w = 0;
    for (int m = 0; m <= truncation; ++m)
      for (int n = m; n <= truncation; ++n) nof[w++] = n;
  }
  // legendre/index.ts:200-221 (kernelTables): grid-to-spectral sums carry
  // skgpsp, spectral-to-grid sums carry skspgp, by total wavenumber n.
  for (auto& kv : tabs) {
    const bool g2s = kv.first == "qc" || kv.first == "qe" || kv.first == "qm" || kv.first == "qq";
    Vec v = kv.second;
    for (size_t i = 0; i < v.size(); ++i) v[i] *= (g2s ? sh.g2s : sh.s2g)[nof[i % modes]];
    sh.q[kv.first] = v;
  }
  return sh;
}

PlanetSetup build_planet(const exogcm_planet& p, const exogcm_boundary& b, const SharedSetup& sh,
                         SetupDevice* device) {
  if (p.star_temperature_k > 0)
    throw std::invalid_argument("stellar-spectrum albedo split (star temperature) is not supported");
  if (p.levels != 5 && p.levels != 10) throw std::invalid_argument("levels must be 5 or 10");
  if (!b.land_mask || !b.t_init || !b.q_init) throw std::invalid_argument("land mask and initial fields required");
  const int T = p.truncation, L = p.levels, nlat = sh.nlat, nlon = sh.nlon, points = nlat * nlon;
  const int nrsp = (T + 1) * (T + 2);
  Pumamod pm = pumamod(p);
  PlanetSetup out;
  out.truncation = T;
  out.levels = L;
  out.filter_kind = p.filter_kind;
  out.filter_gp = p.filter_gp;
  out.filter_sp = p.filter_sp;
  const double tmelt = pm.tmelt;
  const long step = pm.n_start_step;

  // setup/modules/index.ts: the module values this configuration reaches.
  const double co2 = p.co2_ppm;
  const double iyrbp = 1950 - pm.n_start_year;
  (void)iyrbp;
  const double albland = 0.22, dgroundalb = 0.2, doceanalb = 0.069, dsnowalbmn = 0.4, dsnowalbmx = 0.8;
  const double dglacalbmn = 0.6, dicealbmn = 0.5, dicealbmx = 0.7, albsea = 0.069, albice = 0.7;
  const double drhsfull = 0.4, dsmax = 5, wsmax = 0.5, drhsland = 0.25, dz0land = 2, rinifor = 0.5;
  const double albsmaxf1 = 0.5 * dsnowalbmx;
  const double dsoilz[5] = {0.4 * p.soil_depth_scale, 0.8 * p.soil_depth_scale, 1.6 * p.soil_depth_scale,
                            3.2 * p.soil_depth_scale, 6.4 * p.soil_depth_scale};
  const double tfreeze = 271.25, thicec = 0.5;
  const double dz0sea = 1.5e-5, dz0ice = 0.001, drhssea = 1, drhsice = 1;
  const int nglacier = p.glaciers ? 1 : 0;
  const double glacelim = p.glacier_min_depth_m, icesheeth = p.glacier_initial_height_m;
  const double mldepth = p.ocean_depth_m;
  const int nseaice = 1, nice = 1;
  const double gamma = (T == 42 && L == 10) ? 0.007 : 0.01;
  const int freq = (int)std::min<long>(4, pm.mtspd);
  const int interval = (int)(pm.mtspd / freq);
  const double timeweight = 1.0 / (freq * (double)pm.m_days_per_year);
  const double tau_veg = 10 * (double)pm.m_days_per_year * pm.day_24hr;
  const double tau_soil = 42 * (double)pm.m_days_per_year * pm.day_24hr;

  // ---- surfini (setup/surface/index.ts:265-647)
  Vec dls(points), oro(points, 0), dglac(points, 0), dforest(points, rinifor), dwmax(points, std::max(wsmax, 0.0));
  for (int h = 0; h < points; ++h) dls[h] = b.land_mask[h] > 0.5 ? 1 : 0;
  if (b.orography)
    for (int h = 0; h < points; ++h) oro[h] = b.orography[h];
  Vec dtclsoil(points, tmelt), dz0clim(points, dz0land), dz0climo(points, 0);
  Vec dalbcl((size_t)MONTHS * points, albland), dalbcl1((size_t)MONTHS * points, dgroundalb),
      dalbcl2((size_t)MONTHS * points, dgroundalb);
  Vec land_dts(points, 1e20), land_dtsm(points, 1e20), land_dqs(points, 1e20);
  Vec dsoilt((size_t)SOIL * points, tmelt), dsnowt(points, tmelt), dsnowz(points, 0), dwatc(points, 0);
  for (int h = 0; h < points; ++h) {
    if (dls[h] <= 0) continue;
    land_dts[h] = dtclsoil[h];
    for (int l = 0; l < SOIL; ++l) dsoilt[(size_t)l * points + h] = land_dts[h];
    dwatc[h] = drhsland * drhsfull * dwmax[h];
  }
  Vec dalbclim = monthly(dalbcl, step + 1, pm, points), dalbclim1 = monthly(dalbcl1, step + 1, pm, points),
      dalbclim2 = monthly(dalbcl2, step + 1, pm, points);
  if (p.wet_soil) {
    for (int h = 0; h < points; ++h) {
      if (dls[h] <= 0.5) continue;
      if (land_dts[h] > 273.15) {
        const double bf = 0;
        const double al = (1 / 5.2) * std::pow(std::pow(std::max(bf, 1e-3), (1 - 4.0) / 4.0) - 1, 0.25);
        const double dw = std::exp(-std::pow(bf * 25, 6)), ww = std::exp(-std::pow((1 - bf) * 30, 9));
        dalbclim[h] = 0.4 * dw + al * (1 - dw - ww) + doceanalb * ww;
        dalbclim1[h] = dalbclim[h];
        dalbclim2[h] = dalbclim[h];
      } else {
        dalbclim[h] = albland;
        dalbclim1[h] = dgroundalb;
        dalbclim2[h] = dgroundalb;
      }
    }
  }
  Vec dalb(points, 0), dsalb(2 * (size_t)points, 0), drhs(points, 0), dz0(points, 0), dsnow(points, 0);
  Vec soilf[5];
  for (auto& v : soilf) v.assign(points, 0);
  Vec dt((size_t)(L + 1) * points, 0), dq((size_t)(L + 1) * points, 0);
  const size_t sl = (size_t)L * points;
  for (int h = 0; h < points; ++h) {
    if (dls[h] <= 0) continue;
    const double ts = land_dts[h];
    land_dtsm[h] = ts;
    land_dqs[h] = saturation(ts, pm);
    dsnow[h] = dsnowz[h];
    dalb[h] = dalbclim[h];
    dsalb[h] = dalbclim1[h];
    dsalb[points + h] = dalbclim2[h];
    if (dwmax[h] > 0) drhs[h] = std::min(1.0, dwatc[h] / (drhsfull * dwmax[h]));
    dz0[h] = dz0clim[h];
    for (int l = 0; l < SOIL; ++l) soilf[l][h] = dsoilt[(size_t)l * points + h];
    if (dglac[h] > 0.5) {
      dsnowz[h] = std::max(dsmax, 0.0);
      dsnow[h] = dsnowz[h];
      dalb[h] = glacier_albedo(0.8, 0.6, ts, tmelt);
      dsalb[h] = glacier_albedo(dsnowalbmx, dglacalbmn, ts, tmelt);
      dsalb[points + h] = glacier_albedo(dsnowalbmx, dglacalbmn, ts, tmelt);
      drhs[h] = 1;
    }
    dt[sl + h] = ts;
    dq[sl + h] = land_dqs[h];
  }
  if (icesheeth >= 0) {
    for (int h = 0; h < points; ++h) {
      const bool covered = oro[h] != 0;
      dglac[h] = covered ? 1 : 0;
      dsnowz[h] = covered ? icesheeth : 0;
    }
  } else {
    for (int h = 0; h < points; ++h)
      if (dglac[h] > 0 && dsnowz[h] == 0) dsnowz[h] = glacelim;
  }
  Vec doro = oro;
  if (nglacier == 1) {
    const double gm = 6.67408e-11 * 5.9722e24, er = 6.371e6;
    for (int h = 0; h < points; ++h) {
      const double ground = oro[h];
      const double dz = (er * er * ground) / (gm - er * ground);
      const double snow = dsnowz[h] / (850.0 / 1000);
      const double gravity = gm / ((er + dz) * (er + dz));
      doro[h] = ground + (gravity * snow - (gravity / (dz + er)) * snow * snow);
    }
  }
  Vec duroff, dvroff;
  runoff(doro, dls, nlat, nlon, sh.sines, pm, duroff, dvroff);
  Vec so = analyse_planes(sh, doro.data(), 1, device);
  for (double& v : so) v /= (pm.cv * pm.cv);
  if (nglacier == 1)
    for (int h = 0; h < points; ++h)
      if (dsnowz[h] > 30) dglac[h] = 1;
  Vec dpersist(points);
  for (int h = 0; h < points; ++h) dpersist[h] = dls[h] < 0.5 ? 0 : 1;
  for (int h = 0; h < points; ++h)
    if (dls[h] == 0) dforest[h] = 0;
  Vec xls = dls;
  Vec xclsst = surf_field(b.sst, b.sst_months, points, MONTHS, -999);
  Vec xclicec = surf_field(b.ice_cover, b.ice_cover_months, points, MONTHS, -999);
  Vec xcliced((size_t)MONTHS * points, -999);
  {
    const double cover_max = *std::max_element(xclicec.begin(), xclicec.end());
    if (nice >= 0) {
      if (cover_max > 5)
        for (double& v : xclicec) v *= 0.01;
      if (cover_max < 0)
        for (size_t i = 0; i < xclicec.size(); ++i) xclicec[i] = (nice > 0.5 && xclsst[i] <= tfreeze) ? 1 : 0;
      if (xcliced[0] < 0) xcliced = ice_thickness(xclicec, nlat, nlon);
    }
    for (size_t i = 0; i < xclicec.size(); ++i)
      if (nseaice == 0 || xls[i % points] >= 1) {
        xclicec[i] = 0;
        xcliced[i] = 0;
      }
  }
  Vec xclssto = monthly(xclsst, step, pm, points), xclsst2 = monthly(xclsst, step + 1, pm, points);
  Vec xcliced2 = monthly(xcliced, step + 1, pm, points);
  for (double& v : xcliced2) v = std::max(v, 0.0);
  Vec xclicec2 = monthly(xclicec, step + 1, pm, points);
  for (int h = 0; h < points; ++h) xclicec2[h] = xcliced2[h] <= 0 ? 0 : std::max(xclicec2[h], 0.0);
  Vec xiced = xcliced2, xicec(points);
  for (int h = 0; h < points; ++h) xicec[h] = xclicec2[h] >= thicec ? 1 : 0;
  Vec yclsst = surf_field(b.sst, b.sst_months, points, MONTHS, 0);
  for (double& v : yclsst) v = std::max(v, tfreeze);
  Vec yclsst2 = monthly(yclsst, step + 1, pm, points);
  Vec ymld(points, mldepth);
  Vec sea_dts(points, 0), sea_dqs(points, 0), sea_dsst(points, 0), dicec(points, 0), diced(points, 0),
      dmld(points, 0);
  for (int h = 0; h < points; ++h) {
    if (dls[h] >= 0.5) continue;
    const double ts = yclsst2[h];
    sea_dts[h] = ts;
    dicec[h] = xicec[h];
    diced[h] = xiced[h];
    dsnow[h] = 0;
    sea_dsst[h] = ts;
    dmld[h] = ymld[h];
    dt[sl + h] = ts;
    sea_dqs[h] = saturation(ts, pm);
    dq[sl + h] = sea_dqs[h];
    const double c = dicec[h];
    drhs[h] = drhssea * (1 - c) + drhsice * c;
    dalb[h] = albsea * (1 - c) + c * std::min(albice, 0.5 + 0.025 * (273 - ts));
    dsalb[h] = doceanalb * (1 - c) + c * std::min(dicealbmx, dicealbmn + 0.025 * (273 - ts));
    dsalb[points + h] = doceanalb * (1 - c) + c * std::min(dicealbmx, dicealbmn + 0.025 * (273 - ts));
    dz0[h] = dz0sea * (1 - c) + dz0ice * c;
  }
  Vec roww(points);
  for (int h = 0; h < points; ++h) roww[h] = sh.weights[h / nlon];

  // ---- psurf lowered by the mean orography (setup/index.ts:53-62)
  const double mean_height = (so[0] * pm.cv * pm.cv) / std::sqrt(2.0);
  const double psurf_nl = pm.psurf;
  pm.psurf = std::exp(std::log(pm.psurf) - mean_height / pm.gascon / pm.tgr);

  // ---- dynamics set-up and tables
  Dyn dyn = initpm(T, L, pm, pm.akap);
  Vec sr = setzt(dyn, T, pm);
  out.nkits = std::max(pm.nkits, 1);
  if (out.nkits > 3) throw std::invalid_argument("more than 3 start-up steps");
  Vec bm1((size_t)4 * T * L * L, 0), bases((size_t)4 * L * L);
  for (int k = 0; k <= 3; ++k) {
    out.deltsec[k] = pm.day_24hr / pm.mtspd / std::pow(2.0, k);
    out.delt[k] = TWOPI / pm.ntspd / std::pow(2.0, k);
    const Vec base = makebm_base(dyn, out.delt[k]);
    std::copy(base.begin(), base.end(), bases.begin() + (size_t)k * L * L);
  }
  if (device) {
    device->makebm(bases.data(), L, T, bm1.data());
  } else {
    for (int k = 0; k <= 3; ++k) {
      const Vec b1 = makebm(Vec(bases.begin() + (size_t)k * L * L, bases.begin() + (size_t)(k + 1) * L * L), L, T);
      std::copy(b1.begin(), b1.end(), bm1.begin() + (size_t)k * T * L * L);
    }
  }
  auto& tb = out.tables;
  tb["t0"] = dyn.t0;
  tb["dsigma"] = dyn.dsigma;
  tb["sigma"] = dyn.sigma;
  tb["sigmah"] = dyn.sigmah;
  tb["rdsig"] = dyn.rdsig;
  tb["t01s2"] = dyn.t01s2;
  tb["tkp"] = dyn.tkp;
  tb["damp"] = dyn.damp;
  tb["tdisst"] = dyn.tdisst;
  tb["tdissq"] = dyn.tdissq;
  tb["tdissd"] = dyn.tdissd;
  tb["tdissz"] = dyn.tdissz;
  tb["tfrc"] = dyn.tfrc;
  tb["c"] = dyn.c;
  tb["g"] = dyn.g;
  tb["tau"] = dyn.tau;
  tb["bm1"] = bm1;
  tb["sop"] = so;
  tb["srp"] = sr;
  tb["sakpp"] = dyn.sak;
  // physics/surface-flux/index.ts:30-67 (tables)
  {
    const double lamm = 160, vd = 5, zlamh = lamm * std::sqrt(3 * vd * 0.5);
    tb["flux_sigfac"] = {std::pow(dyn.sigma[L - 1], -pm.akap)};
    tb["flux_lnsig"] = {std::log(dyn.sigma[L - 1])};
    Vec skap(L), skaph(L), mixh2(L, 0), mixm2(L, 0), rds(L, 0), sh3(L, 0), kfac(L, 0);
    for (int l = 0; l < L; ++l) {
      skap[l] = std::pow(dyn.sigma[l], pm.akap);
      skaph[l] = std::pow(dyn.sigmah[l], pm.akap);
    }
    for (int l = 0; l < L - 1; ++l) {
      const double zzlev = (-pm.gascon * 250 * std::log(dyn.sigmah[l])) / pm.ga;
      const double zdz = (pm.gascon * 250 * std::log(dyn.sigma[l + 1] / dyn.sigma[l])) / pm.ga;
      const double zmixh = (zlamh * 0.4 * zzlev) / (zlamh + 0.4 * zzlev);
      const double zmixm = (lamm * 0.4 * zzlev) / (lamm + 0.4 * zzlev);
      const double zrdsig = 1 / (dyn.sigma[l + 1] - dyn.sigma[l]);
      mixh2[l] = zmixh * zmixh;
      mixm2[l] = zmixm * zmixm;
      rds[l] = zrdsig;
      sh3[l] = dyn.sigmah[l] * dyn.sigmah[l] * dyn.sigmah[l] * zrdsig;
      const double ratio = (std::pow((zzlev + zdz) / zzlev, 1.0 / 3) - 1) / zdz;
      kfac[l] = std::sqrt(ratio * ratio * ratio / zzlev);
    }
    tb["vdiff_skap"] = skap;
    tb["vdiff_skaph"] = skaph;
    tb["vdiff_mixh2"] = mixh2;
    tb["vdiff_mixm2"] = mixm2;
    tb["vdiff_rdsig"] = rds;
    tb["vdiff_sigmah3"] = sh3;
    tb["vdiff_kfac"] = kfac;
  }
  // physics/radiation/index.ts:59-94 (tables)
  {
    Vec lnsig(L), zzf1(L), zzf3(L);
    lnsig[0] = std::log(dyn.sigma[0] / dyn.sigmah[0]) * 0.5;
    for (int l = 1; l < L; ++l) lnsig[l] = std::log(dyn.sigmah[l - 1] / dyn.sigmah[l]);
    for (int l = 0; l < L; ++l) {
      zzf1[l] = (dyn.sigma[l] * dyn.dsigma[l]) / pm.ga / 100000;
      zzf3[l] = (-1.66 * 0.1 * 1000 * dyn.dsigma[l]) / pm.ga;
    }
    tb["rad_lnsig"] = lnsig;
    tb["lwr_zzf1"] = zzf1;
    tb["lwr_zzf3"] = zzf3;
  }
  // physics/precipitation/index.ts:45-63 (tables)
  {
    Vec rcrit(L), kuo(L, 0);
    for (int l = 0; l < L; ++l)
      rcrit[l] = std::max(0.85, std::max(dyn.sigma[l], 1 - dyn.sigma[l])) * 1.0 *
                 (1 - (2 * 0.0 * (L / 2.0 - (l + 1))) / L);
    for (int l = 0; l < L - 1; ++l) kuo[l] = std::pow(dyn.sigma[l] / dyn.sigma[l + 1], pm.akap);
    tb["rcrit"] = rcrit;
    tb["kuo_zfac"] = kuo;
  }
  tb["dsoilz"] = Vec(dsoilz, dsoilz + 5);

  // ---- constants (setup/index.ts:53-375), by WGSL override name
  auto& k = out.consts;
  const double tswr1 = 0.077, tswr2 = 0.065, tswr3 = 0.0055;
  const double zao30 = 0.209 * std::pow(7e-5, 0.436), zco20 = 0.0676 * std::pow(0.01022, 0.421);
  const double zh2o0a = 0.846 * std::pow(3.59e-5, 0.243), zh2o0 = 0.832 * std::pow(0.0286, 0.26);
  int jet = 0;
  for (int l = 1; l < L; ++l)
    if (std::fabs(dyn.sigma[l] - 0.25) < std::fabs(dyn.sigma[jet] - 0.25)) jet = l;
  k = {
      {"PSURF", pm.psurf}, {"WW", pm.ww}, {"CV", pm.cv}, {"CT", pm.ct}, {"AKAP", pm.akap}, {"RDBRV", pm.rdbrv},
      {"ADV", pm.adv}, {"ACPD", pm.acpd}, {"GA", pm.ga}, {"GASCON", pm.gascon}, {"PLAVOR", pm.plavor},
      {"PNU", pm.pnu}, {"PNU21", pm.pnu21}, {"RA1", pm.ra1}, {"RA2", pm.ra2}, {"RA4", pm.ra4},
      {"TMELT", pm.tmelt}, {"ALV", pm.alv}, {"ALS", pm.als}, {"MOIST", 1 / pm.rdbrv - 1}, {"ZUMIN", 1},
      {"VDIFF_B", 5}, {"VDIFF_C", 5}, {"VDIFF_D", 5}, {"NDHEAT", pm.ndheat > 0 ? 1 : 0},
      {"NFIXED", p.synchronous ? 1 : 0}, {"ZRLON", TWOPI / nlon}, {"ZDAWN", 0}, {"OZONE", p.ozone ? 1 : 0},
      {"A0O3", 0.25}, {"A1O3", 0.11}, {"ACO3", 0.08}, {"BO3", 20000}, {"CO3", 5000},
      {"ZCONST", std::exp(-20000.0 / 5000.0)}, {"GSOL0", pm.gsol0}, {"ZSOLAR1", 0.517}, {"ZSOLAR2", 0.483},
      {"ZSOLARS1", 0}, {"ZSOLARS2", 0}, {"TSWR1", tswr1}, {"TSWR2", tswr2}, {"TSWR3", tswr3},
      {"ZB3", (tswr1 * std::sqrt(0.5)) / 0.5}, {"ZB4", tswr2 * std::sqrt(0.5)}, {"ZB5", tswr3 * 0.25},
      {"RCOEFF", 1}, {"LN_DIFFUSE_RAYLEIGH", std::log(1 - 0.144)}, {"NSTARTEMP", 0}, {"SBK", SBK},
      {"TH2OC", 0.024}, {"TPOFMT", 1}, {"ZFCO2_ZZF2", (100 / 1.9635) * (0.0440098 / 0.0289644) * 1e-6},
      {"ZAO30", zao30}, {"ZCO20", zco20}, {"ZH2O0A", zh2o0a}, {"ZH2O0", zh2o0},
      {"ZAO3C", 0.209 * std::pow(0.01 + 7e-5, 0.436) - zao30 - 0.0212 * std::log10(0.01)},
      {"ZACO2C", 0.0676 * std::pow(1.01022, 0.421) - zco20},
      {"ZAH2OC", 0.846 * std::pow(0.01 + 3.59e-5, 0.243) - zh2o0a - 0.24 * std::log10(0.02)},
      {"ZTH2OC", 1 - (0.832 * std::pow(2 + 0.0286, 0.26) - zh2o0) + 0.1196 * std::log(2 - 0.6931)},
      {"RHBETA", 0}, {"NBETA", 3}, {"PDEEP", 999999}, {"PDEEPTH", 70000}, {"RKSHALLOW", 10}, {"GAMMA", gamma},
      {"ZRFAC", pm.solar_day * 1000}, {"CLWFAC", 1 / (-0.1 - 0.0) < 0 ? -1.0 : 1.0}, {"CLWCRIT1", -0.1},
      {"CLWCRIT2", 0}, {"SICECAP", 2.07e6}, {"SOILCAP", 2.4e6}, {"SICEDIFF", 2.03}, {"SOILDIFF", 1.8},
      {"SNOWCAP", 0.6897e6}, {"SNOWDIFF", 0.31}, {"RHOSNOW", 330}, {"DZTOP", 0.2}, {"DSMAX", dsmax},
      {"ALBSMAX", 0.8}, {"ALBSMIN", 0.4}, {"ALBSMAXF", 0.4}, {"ALBSMINF", 0.3}, {"ALBSMAX1", dsnowalbmx},
      {"ALBSMIN1", dsnowalbmn}, {"ALBSMAXF1", albsmaxf1}, {"ALBSMINF1", 0.75 * albsmaxf1}, {"ALBSMAX2", dsnowalbmx},
      {"ALBSMIN2", dsnowalbmn}, {"ALBSMAXF2", albsmaxf1}, {"ALBSMINF2", 0.75 * albsmaxf1}, {"ALBGMAX", 0.8},
      {"ALBGMIN", 0.6}, {"ALBGMAX1", dsnowalbmx}, {"ALBGMIN1", dglacalbmn}, {"ALBGMAX2", dsnowalbmx},
      {"ALBGMIN2", dglacalbmn}, {"DRHSFULL", drhsfull}, {"NWETSOIL", p.wet_soil ? 1 : 0}, {"WSMAX", wsmax},
      {"ALBLAND", albland}, {"ALBLANDMAX", 0.4}, {"DGROUNDALB1", dgroundalb}, {"DGROUNDALB2", dgroundalb},
      {"DOCEANALB1", doceanalb}, {"DOCEANALB2", doceanalb}, {"NVEG", (double)pm.nveg}, {"RLUE", 3.4e-10},
      {"CO2CONV", 8.3e-4}, {"TAU_VEG", tau_veg}, {"TAU_SOIL", tau_soil}, {"VWS_CRIT", 0.25}, {"Q10", 2},
      {"ZLAIMAX", 9}, {"ZLAIMIN", 0.1}, {"VALB_MIN", 0.12}, {"VALB_MAX", 0.3}, {"VSALB_MIN", 0.2},
      {"VWMAX_MAX", 0.5}, {"VWMAX_MIN", 0.05}, {"VZ0_MIN", 0.05}, {"CVEG_A", 2.9}, {"CVEG_C", 1.570796326794897},
      {"CVEG_F", 3}, {"CVEG_K", 0.5}, {"CVEG_L", 0.25}, {"CT_CRIT", 5}, {"CO2_REF", 360}, {"CO2_COMP", 0},
      {"CO2_SENS", 0.3}, {"CVEG_E", std::atan(-1.9)}, {"CVEG_G", std::atan(-3.0)}, {"NCVEG", 1},
      {"NGLACIER", nglacier ? 1.0 : 0.0}, {"GLACELIM", glacelim}, {"XDT", pm.solar_day / pm.ntspd},
      {"XMIND", 0.1}, {"XMAXD", 9}, {"CICEMIN", 0.5}, {"THICEC", thicec}, {"TFREEZE", tfreeze},
      {"CRHOI", 920}, {"CRHOS", 1030}, {"CRHOSN", 330}, {"CPI", 2070}, {"CKAPI", 2.03}, {"CKAPSN", 0.31},
      {"CLFI", 3.28e5}, {"CLFSN", 3.337e5}, {"DTMIX", pm.solar_day / pm.ntspd}, {"CPS", 4180},
      {"CHARNOCK", 0.018}, {"DZ0SEA", dz0sea}, {"DZ0ICE", dz0ice}, {"DRHSSEA", drhssea}, {"DRHSICE", drhsice},
      {"ALBSEA", albsea}, {"ALBICE", albice}, {"DICEALBMX1", dicealbmx}, {"DICEALBMX2", dicealbmx},
      {"DICEALBMN1", dicealbmn}, {"DICEALBMN2", dicealbmn}, {"NCARBON", 1}, {"NSUPPLY", 0},
      {"TIMEWEIGHT", timeweight}, {"CO2EARTH", 330}, {"BETA", 0.5}, {"KACT", 0.09}, {"PEARTH", 79},
      {"WMAX", 80.9}, {"VEARTH", 0.05}, {"PLARAD", pm.plarad}, {"RAD_EARTHSQ", 6371220.0 * 6371220.0},
      {"JET", (double)jet}, {"SIGMA_LOW", dyn.sigma[L - 1]},
  };
  // rainini's clwfac with the default clwcrit1 = -0.1 < clwcrit2 = 0.
  k["CLWFAC"] = -1.0;
  // hurricane_namelist (setup/index.ts:107-113; defaults CKCD 0.9, VITHRESH
  // 0.145); RD and OMEGA are GASCON and WW.
  k["NSTORMDIAG"] = p.storm_diagnostics ? 1 : 0;
  k["CKCD"] = p.storm_ckcd > 0 ? p.storm_ckcd : 0.9;
  k["VITHRESH"] = p.storm_vithresh > 0 ? p.storm_vithresh : 0.145;

  // ---- initial state: the synthetic atmosphere transformed in f64, plus surfini's fields
  auto& st = out.state;
  Vec stv((size_t)L * nrsp, 0), sqv((size_t)L * nrsp, 0), szv((size_t)L * nrsp, 0);
  {
    // The L temperature planes then the L humidity planes, analysed together.
    Vec grids((size_t)2 * L * points);
    for (int l = 0; l < L; ++l)
      for (int h = 0; h < points; ++h)
        grids[(size_t)l * points + h] = b.t_init[(size_t)l * points + h] / pm.ct - dyn.t0[l];
    std::copy(b.q_init, b.q_init + (size_t)L * points, grids.begin() + (size_t)L * points);
    const Vec spec = analyse_planes(sh, grids.data(), 2 * L, device);
    std::copy(spec.begin(), spec.begin() + (size_t)L * nrsp, stv.begin());
    std::copy(spec.begin() + (size_t)L * nrsp, spec.end(), sqv.begin());
    for (int l = 0; l < L; ++l) szv[(size_t)l * nrsp + 2] = pm.plavor;
  }
  Vec spv(nrsp, 0);
  st["sp"] = spv;
  st["spm"] = std::move(spv);
  st["st"] = stv;
  st["stm"] = std::move(stv);
  st["sz"] = szv;
  st["szm"] = std::move(szv);
  st["sd"] = Vec((size_t)L * nrsp, 0);
  st["sdm"] = Vec((size_t)L * nrsp, 0);
  st["sq"] = sqv;
  st["sqm"] = std::move(sqv);
  st["dls"] = dls;
  st["dz0"] = std::move(dz0);
  st["drhs"] = std::move(drhs);
  st["dwatc"] = std::move(dwatc);
  st["dqco2"] = Vec((size_t)L * points, co2 > 0 ? co2 : 0);
  st["co2"] = {co2};
  st["dalb"] = std::move(dalb);
  st["dsalb"] = std::move(dsalb);
  st["dicec"] = std::move(dicec);
  st["diced"] = std::move(diced);
  st["dmld"] = std::move(dmld);
  st["dforest"] = std::move(dforest);
  st["dglac"] = std::move(dglac);
  st["dpersist"] = std::move(dpersist);
  st["dwmax"] = std::move(dwmax);
  st["dsnow"] = std::move(dsnow);
  st["dtsoil"] = soilf[0];
  st["dtd2"] = soilf[1];
  st["dtd3"] = soilf[2];
  st["dtd4"] = soilf[3];
  st["dtd5"] = soilf[4];
  st["dt"] = std::move(dt);
  st["dq"] = std::move(dq);
  st["land_dts"] = std::move(land_dts);
  st["land_dtsm"] = std::move(land_dtsm);
  st["land_dqs"] = std::move(land_dqs);
  st["duroff"] = std::move(duroff);
  st["dvroff"] = std::move(dvroff);
  st["darea"] = roww;
  st["dsnowt"] = std::move(dsnowt);
  st["dsnowz"] = std::move(dsnowz);
  st["dz0climo"] = std::move(dz0climo);
  st["dalbclim"] = std::move(dalbclim);
  st["dalbclim1"] = std::move(dalbclim1);
  st["dalbclim2"] = std::move(dalbclim2);
  st["dsoilt"] = std::move(dsoilt);
  st["dalbcl"] = std::move(dalbcl);
  st["dalbcl1"] = std::move(dalbcl1);
  st["dalbcl2"] = std::move(dalbcl2);
  st["dagg"] = Vec(points, p.initial_growth);
  st["dgrow"] = Vec(points, 1.0);
  st["dsc"] = Vec(points, 1.0);
  st["dmr"] = Vec(points, 2.0);
  st["xts"] = yclsst2;
  st["xsst"] = yclsst2;
  st["xmld"] = ymld;
  st["xls"] = std::move(xls);
  st["xiced"] = std::move(xiced);
  st["xicec"] = std::move(xicec);
  st["xgw"] = std::move(roww);
  st["xclsst2"] = std::move(xclsst2);
  st["xclicec2"] = std::move(xclicec2);
  st["xcliced2"] = std::move(xcliced2);
  st["xclssto"] = std::move(xclssto);
  st["xclsst"] = std::move(xclsst);
  st["xclicec"] = std::move(xclicec);
  st["xcliced"] = std::move(xcliced);
  st["ysst"] = yclsst2;
  st["ymld"] = std::move(ymld);
  st["yls"] = std::move(dls);
  st["yclsst2"] = std::move(yclsst2);
  st["yclsst"] = std::move(yclsst);
  st["sea_dts"] = std::move(sea_dts);
  st["sea_dqs"] = std::move(sea_dqs);
  st["sea_dsst"] = std::move(sea_dsst);
  (void)psurf_nl;

  // ---- calendar (setup/index.ts:304-318, calendar/index.ts:37-126 for a fixed orbit)
  if (!p.fixed_orbit) throw std::invalid_argument("only a fixed orbit is supported (NFIXORB = 1)");
  {
    const double pi = 4 * std::atan(1.0), degrad = pi / 180;
    Calendar& c = out.cal;
    Orbit& o = c.orbit;
    const double e = pm.eccen, e2 = e * e, e3 = e2 * e;
    const double mvelpp = (pm.mvelp + 180) * degrad, beta = std::sqrt(1 - e2);
    o.eccentricity = e;
    o.obliquity_rad = pm.obliq * degrad;
    o.mean_anomaly_rad = pm.meananom0 * degrad;
    o.perihelion_longitude_rad = mvelpp;
    o.mean_longitude_at_equinox_rad =
        2 * ((0.5 * e + 0.125 * e3) * (1 + beta) * std::sin(mvelpp) - 0.25 * e2 * (0.5 + beta) * std::sin(2 * mvelpp) +
             0.125 * e3 * (1.0 / 3 + beta) * std::sin(3 * mvelpp));
    c.keplerian = p.keplerian != 0;
    c.fixed_sun = p.synchronous != 0;
    c.fixed_longitude_deg = pm.fixedlon;
    c.fixed_declination_rad = o.obliquity_rad;
    c.steps_per_year = pm.n_steps_per_year;
    c.steps_per_day = pm.ntspd;
    c.output_window_steps = pm.nafter;
    c.step_minutes = pm.mpstep;
    c.days_per_year = pm.n_days_per_year;
    c.days_per_month = pm.n_days_per_month;
    c.solar_day = pm.solar_day;
    c.rotation_speed = pm.rotspd;
    c.toffo3 = 0.25;
    c.carbon_interval = interval;
  }
  out.start_step = pm.n_start_step;
  return out;
}

// stepper/index.ts:281-334 (values) with calendar/solar/index.ts:26-89,
// radiation/index.ts:96-113, surface/index.ts:49-59 and carbon/index.ts:23-28.
void calendar_date(const Calendar& cal, long step, int out[5]) {
  const Date d = cal_date(step, cal.steps_per_day, cal.days_per_year, cal.step_minutes);
  out[0] = (int)d.year;
  out[1] = d.month;
  out[2] = d.day;
  out[3] = d.hour;
  out[4] = d.minute;
}

StepValues step_values(const Calendar& cal, long step, int carbon_step) {
  StepValues v{};
  const double calendar_day = (double)(step % cal.steps_per_year) / cal.steps_per_year;
  const long minutes = trunc_l((double)(step % cal.steps_per_day) * cal.step_minutes);
  const Orbit& o = cal.orbit;
  const double e = o.eccentricity;
  double longitude, distance;
  if (cal.keplerian) {
    double true_anomaly = 0;
    distance = 1;
    if (!cal.fixed_sun) {
      double mean = calendar_day * TWOPI + o.mean_anomaly_rad;
      while (mean > TWOPI) mean -= TWOPI;
      while (mean < 0) mean += TWOPI;
      if (e > 0) {
        double value = e < 0.5 ? mean : PI;
        for (int it = 0; it < 101; ++it) {
          const double prev = value;
          value -= (value - (mean + e * std::sin(value))) / std::max(1e-15, 1 - e * std::cos(value));
          if (std::fabs(value - prev) <= 1e-14) break;
        }
        const double tangent = std::tan(value * 0.5);
        const double mag = std::sqrt(((1 + e) / (1 - e)) * tangent * tangent);
        true_anomaly = 2 * std::atan(tangent < 0 ? -mag : mag);
        if (true_anomaly < 0) true_anomaly += TWOPI;
        true_anomaly = std::fmod(true_anomaly, TWOPI);
        const double inv = 1 / (1 - e * std::cos(value));
        distance = inv * inv;
      } else {
        true_anomaly = mean;
      }
    }
    longitude = std::fmod(o.perihelion_longitude_rad + true_anomaly, TWOPI);
  } else {
    const double ml = o.mean_longitude_at_equinox_rad + (calendar_day - 80.5 / 365) * 2 * M_PI;
    const double anomaly = ml - o.perihelion_longitude_rad;
    const double sine = std::sin(anomaly);
    longitude = ml + e * (2 * sine + e * (1.25 * std::sin(2 * anomaly) + e * ((13.0 / 12) * std::sin(3 * anomaly) - 0.25 * sine)));
    const double inv = (1 + e * std::cos(longitude - o.perihelion_longitude_rad)) / (1 - e * e);
    distance = inv * inv;
  }
  const double declination_orbit = std::asin(std::sin(o.obliquity_rad) * std::sin(longitude));
  const double right_ascension =
      std::atan2(std::cos(o.obliquity_rad) * std::sin(longitude), std::cos(longitude));
  const double declination = cal.fixed_sun ? cal.fixed_declination_rad : declination_orbit;
  const double phase = cal.fixed_sun ? (1 - cal.fixed_longitude_deg / 360) * TWOPI
                                     : ((double)minutes * cal.rotation_speed * TWOPI) / 1440;
  v.rad[0] = std::sin(declination);
  v.rad[1] = std::cos(declination);
  v.rad[2] = phase - (cal.keplerian ? right_ascension : 0);
  v.rad[3] = distance;
  v.rad[4] = std::cos(TWOPI * (calendar_day - cal.toffo3));
  double now[3], nx[3];
  month_interp(step, cal.steps_per_day, cal.days_per_year, cal.days_per_month, cal.step_minutes, cal.solar_day, now);
  month_interp(step + 1, cal.steps_per_day, cal.days_per_year, cal.days_per_month, cal.step_minutes, cal.solar_day,
               nx);
  const long y0 = cal_date(step, cal.steps_per_day, cal.days_per_year, cal.step_minutes).year;
  const long y1 = cal_date(step + 1, cal.steps_per_day, cal.days_per_year, cal.step_minutes).year;
  for (int i = 0; i < 3; ++i) {
    v.surf[i] = now[i];
    v.surf[3 + i] = nx[i];
  }
  v.surf[6] = y1 != y0 ? 1 : 0;
  const int next = carbon_step + 1;
  const bool weathers = next == cal.carbon_interval;
  v.carbon = weathers ? 1 : 0;
  v.next_carbon_step = weathers ? 0 : next;
  return v;
}

}  // namespace exogcm
