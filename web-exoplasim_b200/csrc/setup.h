// Host-side FP64 set-up of one planet: the reference's SETUP (pumamod, the
// physics modules' *ini, initpm/initsi/makebm/setzt, surfini) and CALENDAR.
#pragma once
#include <map>
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

SharedSetup build_shared(int truncation, int filter_kind, int filter_gp, int filter_sp);
PlanetSetup build_planet(const exogcm_planet& planet, const exogcm_boundary& boundary, const SharedSetup& shared);
StepValues step_values(const Calendar& cal, long step, int carbon_step);

}  // namespace exogcm
