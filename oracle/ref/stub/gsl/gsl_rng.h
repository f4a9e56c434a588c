/* Stand-in for GSL's default generator, which is MT19937 (GSL manual, "Random
 * number generator algorithms"): seeded by the standard MT19937 initialisation
 * with seed 0 mapped to 4357, uniform doubles = 32-bit output / 2^32.
 * std::mt19937 implements the same published recurrence and seeding.  Real GSL
 * is not installed here, so bit-equality with libgsl is unverified; the harness
 * only uses this generator where the reference itself draws random numbers
 * (Ritz start vectors, FERMIONS/OVERLAP/OverlapUpdate.cpp:66-84). */
#pragma once
#include <random>
#include <cstdint>
typedef struct { std::mt19937 engine; unsigned long draws; } gsl_rng;
typedef int gsl_rng_type;
static const gsl_rng_type *gsl_rng_default = nullptr;
static inline void gsl_rng_env_setup() {}
static inline gsl_rng *gsl_rng_alloc(const gsl_rng_type *) { gsl_rng *r = new gsl_rng; r->draws = 0; return r; }
static inline void gsl_rng_set(gsl_rng *r, unsigned long s) { r->engine.seed((uint32_t)(s == 0 ? 4357UL : s)); r->draws = 0; }
static inline double gsl_rng_uniform(gsl_rng *r) { r->draws++; return (double)r->engine() / 4294967296.0; }
static inline double gsl_rng_uniform_pos(gsl_rng *r) { double u; do { u = gsl_rng_uniform(r); } while (u == 0.0); return u; }
