// Host-side FP64 set-up of one planet: the reference's SETUP (pumamod, the
// physics modules' *ini, initpm/initsi/makebm/setzt, surfini) and CALENDAR.
#pragma once
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/exogcm.h"

namespace exogcm {

using Vec = std::vector<double>;

// Per-step host values (stepper/index.ts:281-334).
struct StepValues {
  double rad[5];
  double surf[7];
  double carbon;
  int next_carbon_step;
};

struct Orbit {
  double eccentricity, obliquity_rad, perihelion_longitude_rad, mean_anomaly_rad, mean_longitude_at_equinox_rad;
};

struct Calendar {
  bool keplerian;
  bool fixed_sun;
  double fixed_longitude_deg, fixed_declination_rad;
  long steps_per_year;
  long steps_per_day;
  long output_window_steps;
  double step_minutes;
  long days_per_year;
  long days_per_month;
  double solar_day;
  double rotation_speed;
  double toffo3;
  Orbit orbit;
  int carbon_interval;
};

// Shared tables of one resolution and filter setting.
struct SharedSetup {
  int truncation, nlat, nlon;
  Vec sines, weights;
  Vec fwd, inv;                     // Fourier tables
  std::map<std::string, Vec> q;     // legendre_q* [NLAT][NCSP], filtered
  Vec qc_unfiltered;                // for set-up analysis
  Vec g2s, s2g;                     // filters by total wavenumber
};

struct PlanetSetup {
  int truncation, levels, nkits;
  long start_step;
  std::map<std::string, double> consts;           // PlanetConst values by name
  double deltsec[4], delt[4];                      // timesteps per phase (kits 0..3)
  std::map<std::string, Vec> tables;               // per-planet tables (bm1 holds 4 phases)
  std::map<std::string, Vec> state;                // initial state fields, reference layout
  Calendar cal;
  int filter_kind, filter_gp, filter_sp;
};

// The set-up's heavy FP64 loops on a device (setup_device.cu). Each call
// keeps the host loop's order of operations and is compiled without
// multiply-add contraction, so it returns the host's numbers bit for bit.
class SetupDevice {
 public:
  virtual ~SetupDevice() = default;
  // legini and the filters of one resolution (legendre/index.ts:29-136):
  // the eight filtered tables [lat][mode] into `q` and the unfiltered qc.
  virtual void legini(const Vec& sines, const Vec& weights, int truncation, const Vec& g2s, const Vec& s2g,
                      std::map<std::string, Vec>& q, Vec& qc_unfiltered) = 0;
  // Grid -> spectral for `planes` grids [plane][lat][lon] in FP64
  // (fourier/index.ts:95-115 then legendre/index.ts:334-361) into
  // `spectra` [plane][2 * modes].
  virtual void analyse(const SharedSetup& shared, const double* grids, int planes, double* spectra) = 0;
  // makebm's inverses (dynamics/setup/index.ts:154-239) of the four phases:
  // `base` holds each phase's n x n matrix before the diagonal term, `bm1`
  // receives [phase][degree - 1][n][n].
  virtual void makebm(const double* base, int n, int truncation, double* bm1) = 0;
};

// A set-up device on the current CUDA device (nullptr-free; throws on a
// CUDA error).
std::unique_ptr<SetupDevice> make_setup_device();

// With `device` null every loop runs on the host.
SharedSetup build_shared(int truncation, int filter_kind, int filter_gp, int filter_sp, SetupDevice* device = nullptr);
PlanetSetup build_planet(const exogcm_planet& planet, const exogcm_boundary& boundary, const SharedSetup& shared,
                         SetupDevice* device = nullptr);
StepValues step_values(const Calendar& cal, long step, int carbon_step);
// The calendar date of a model step (calendar/date/index.ts:43-80):
// year, month, day, hour, minute.
void calendar_date(const Calendar& cal, long step, int out[5]);

}  // namespace exogcm
