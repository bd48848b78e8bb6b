/*
 * Case definitions shared by the two oracle harnesses (ref_fixture.c over
 * the reference library, gcs_oracle.c over the restatement) and mirrored by
 * the device case builder, so that all three construct identical inputs.
 * Test infrastructure.
 */
#ifndef GCS_ORACLE_CASES_COMMON_H
#define GCS_ORACLE_CASES_COMMON_H

#include <math.h>
#include <stdint.h>

enum { CASE_UNIFORM = 0, CASE_SHOCK = 1, CASE_WIND = 2, CASE_PULSE = 3 };

/* Code units of the reference Earth driver: x in R_E, u in 100 km/s,
 * rho in proton cm^-3 (cubedsphere/tests/test_cubedsphere_dipole_background.c
 * :282-294, 467-471). */
#define CASE_RHO_NORM 1.67262192369e-21
#define CASE_DIPOLE_MOMENT (-6761.730688424097)

static inline double case_magnetic_norm_tesla(void) {
  return 100000.0 * sqrt(4.0e-7 * acos(-1.0) * CASE_RHO_NORM);
}

static inline uint64_t case_splitmix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}

/* Uniform in [-1, 1), from the seed, face and storage cell index only. */
static inline double case_noise(unsigned long long seed, int face,
                                size_t cell) {
  const uint64_t h = case_splitmix64(case_splitmix64((uint64_t)seed) ^
                                     ((uint64_t)face << 56) ^ (uint64_t)cell);
  return 2.0 * ((double)(h >> 11) * 0x1.0p-53) - 1.0;
}

/* Wind parameters: n = 5 cm^-3, T = 1e5 K (protons), IMF Bz = -5 nT,
 * V = -400 km/s (CASE_WIND) or -450 km/s with a 20 % sinusoidal density
 * pulse of wavelength 10 R_E along x (CASE_PULSE). */
static inline double case_wind_pressure(void) {
  return 5.0e6 * 1.380649e-23 * 1.0e5 / (CASE_RHO_NORM * 1.0e10);
}

/* An explicit upstream driver (n in cm^-3, Vx in km/s, T in K, Bz in nT)
 * in code units: the density before noise, Vx, pressure n k T and Bz.  No
 * reference counterpart: the reference driver fixes the values above. */
typedef struct {
  double rho, vx, pres, bz;
} case_driver;

static inline case_driver case_driver_code_units(double density_cm3, double vx_kms,
                                                 double temperature_k, double bz_nt) {
  case_driver d;
  d.rho = density_cm3;
  d.vx = vx_kms / 100.0;
  d.pres = density_cm3 * 1.0e6 * 1.380649e-23 * temperature_k / (CASE_RHO_NORM * 1.0e10);
  d.bz = bz_nt * 1.0e-9 / case_magnetic_norm_tesla();
  return d;
}

static inline double case_wind_density(int kind, unsigned long long seed,
                                       int face, size_t cell, double x) {
  double rho = 5.0 * (1.0 + 0.01 * case_noise(seed, face, cell));
  if (kind == CASE_PULSE) rho *= 1.0 + 0.2 * sin(2.0 * acos(-1.0) * x / 10.0);
  return rho;
}

#endif
